// Config: the radiation.cfg grammar of the reference (Config.cpp:8-131,
// Config.h:4-48), kept line-compatible, with additive keys.
//
// Grammar (one item per line; lines starting with '#' and empty lines are
// skipped; lines matching no key are ignored, as in the reference):
//   numregs = N            must precede any [region] section
//   meshfile = <rest of line>
//   outfile = <rest of line>          (default solution.vtk)
//   angorder = maxk   device = d   soltype = s   dump = 0|1
//   precondition = 0|1
//   [region r]  then  kappa = x   Ip = x        (0 <= r <= numregs)
// Additive keys (ignored by the reference, default-initialised here):
//   any "key = value" line outside a section is kept as a string and can be
//   read with get_string/get_int/get_double (e.g. tolerance, maxiter, mode);
//   inside a section likewise per region (e.g. albedo = 0.999).
// Differences: errors raise ConfigError instead of `throw 0`; maxk, prec
// and soltype default to 1, 0, 0 instead of being left uninitialised; the
// trailing newline of meshfile/outfile is removed only if present.
#pragma once
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace transfer {

struct ConfigError : public std::runtime_error {
    explicit ConfigError(const std::string &m) : std::runtime_error(m) {}
};

class Config {
public:
    explicit Config(const char *cfgfile);
    double getKappa(int region) const { return kappa_.at(region); }
    double getIp(int region) const { return Ip_.at(region); }
    const char *getMeshFilename() const { return meshfn_.c_str(); }
    const char *getOutFilename() const { return outfn_.c_str(); }
    int getMaxK() const { return maxk_; }
    int getDevice() const { return dev_; }
    bool doDump() const { return dump_ != 0; }
    bool usePrec() const { return prec_ != 0; }
    int solType() const { return soltype_; }
    int numRegions() const { return nreg_; }

    bool has(const std::string &key) const { return extra_.count(key) != 0; }
    std::string get_string(const std::string &key, const std::string &dflt = "") const;
    double get_double(const std::string &key, double dflt) const;
    int get_int(const std::string &key, int dflt) const;
    bool region_has(int region, const std::string &key) const;
    double region_double(int region, const std::string &key, double dflt) const;

private:
    int nreg_ = -1, maxk_ = 1, dev_ = 0, dump_ = 0, prec_ = 0, soltype_ = 0;
    std::vector<double> kappa_, Ip_;
    std::string meshfn_, outfn_ = "solution.vtk";
    std::map<std::string, std::string> extra_;
    std::vector<std::map<std::string, std::string> > region_extra_;
};

}  // namespace transfer
