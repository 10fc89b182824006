// Config parser (see config.h).
#include "config.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>

namespace transfer {

static std::string trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

Config::Config(const char *cfgfile) {
    FILE *f = std::fopen(cfgfile, "r");
    if (!f) throw ConfigError(std::string("failed to open file `") + cfgfile + "'");
    char buf[1024];
    int line = 0, rid = -1;
    auto die = [&](const std::string &msg) {
        std::fclose(f);
        std::ostringstream os;
        os << cfgfile << ":" << line << ": " << msg;
        throw ConfigError(os.str());
    };
    auto strip_nl = [](char *b) {
        size_t n = std::strlen(b);
        while (n && (b[n - 1] == '\n' || b[n - 1] == '\r')) b[--n] = 0;
    };
    while (std::fgets(buf, sizeof buf, f)) {
        line++;
        if (buf[0] == '#' || buf[0] == '\n') continue;
        if (buf[0] == '[') {
            if (std::sscanf(buf, "[region %d]", &rid) != 1) die("scanf failed to parse region section");
            if (nreg_ < 0) die("section appeared before numregs was set");
            if (rid > nreg_ || rid < 0) die("region id is out of bounds");
            continue;
        }
        if (!std::strncmp(buf, "kappa", 5)) {
            if (rid < 0) die("kappa parameter outside section");
            if (std::sscanf(buf, "kappa = %lf", &kappa_[rid]) != 1) die("scanf failed to parse kappa parameter");
            continue;
        }
        if (!std::strncmp(buf, "Ip", 2)) {
            if (rid < 0) die("Ip parameter outside section");
            if (std::sscanf(buf, "Ip = %lf", &Ip_[rid]) != 1) die("scanf failed to parse Ip parameter");
            continue;
        }
        if (!std::strncmp(buf, "meshfile = ", 11)) {
            if (rid >= 0) die("meshfile parameter in section");
            strip_nl(buf);
            meshfn_ = std::string(buf + 11);
            continue;
        }
        if (!std::strncmp(buf, "outfile = ", 10)) {
            if (rid >= 0) die("outfile parameter in section");
            strip_nl(buf);
            outfn_ = std::string(buf + 10);
            continue;
        }
        if (!std::strncmp(buf, "numregs", 7)) {
            if (rid >= 0) die("numregs parameter in section");
            if (std::sscanf(buf, "numregs = %d", &nreg_) != 1) die("scanf failed to parse numregs parameter");
            if (nreg_ < 0 || nreg_ > 1000000) die("numregs out of range");
            kappa_.assign(nreg_ + 1, 0.0);
            Ip_.assign(nreg_ + 1, 0.0);
            region_extra_.assign(nreg_ + 1, std::map<std::string, std::string>());
            continue;
        }
        if (!std::strncmp(buf, "angorder", 8)) {
            if (rid >= 0) die("angorder parameter in section");
            if (std::sscanf(buf, "angorder = %d", &maxk_) != 1) die("scanf failed to parse angorder parameter");
            continue;
        }
        if (!std::strncmp(buf, "device", 6)) {
            if (rid >= 0) die("device parameter in section");
            if (std::sscanf(buf, "device = %d", &dev_) != 1) die("scanf failed to parse device parameter");
            continue;
        }
        if (!std::strncmp(buf, "soltype", 7)) {
            if (rid >= 0) die("soltype parameter in section");
            if (std::sscanf(buf, "soltype = %d", &soltype_) != 1) die("scanf failed to parse soltype parameter");
            continue;
        }
        if (!std::strncmp(buf, "dump", 4)) {
            if (rid >= 0) die("dump parameter in section");
            if (std::sscanf(buf, "dump = %d", &dump_) != 1) die("scanf failed to parse dump parameter");
            continue;
        }
        if (!std::strncmp(buf, "precondition", 12)) {
            if (rid >= 0) die("precondition parameter in section");
            if (std::sscanf(buf, "precondition = %d", &prec_) != 1)
                die("scanf failed to parse precondition parameter");
            continue;
        }
        // additive "key = value" lines (silently ignored by the reference)
        std::string s(buf);
        size_t eq = s.find('=');
        if (eq == std::string::npos) continue;
        std::string key = trim(s.substr(0, eq)), val = trim(s.substr(eq + 1));
        if (key.empty()) continue;
        if (rid >= 0) region_extra_[rid][key] = val;
        else extra_[key] = val;
    }
    std::fclose(f);
}

std::string Config::get_string(const std::string &key, const std::string &dflt) const {
    auto it = extra_.find(key);
    return it == extra_.end() ? dflt : it->second;
}
double Config::get_double(const std::string &key, double dflt) const {
    auto it = extra_.find(key);
    if (it == extra_.end()) return dflt;
    char *end = nullptr;
    double v = std::strtod(it->second.c_str(), &end);
    if (end == it->second.c_str()) throw ConfigError("bad numeric value for " + key);
    return v;
}
int Config::get_int(const std::string &key, int dflt) const {
    auto it = extra_.find(key);
    if (it == extra_.end()) return dflt;
    char *end = nullptr;
    long v = std::strtol(it->second.c_str(), &end, 10);
    if (end == it->second.c_str()) throw ConfigError("bad integer value for " + key);
    return static_cast<int>(v);
}
bool Config::region_has(int region, const std::string &key) const {
    if (region < 0 || region >= static_cast<int>(region_extra_.size())) return false;
    return region_extra_[region].count(key) != 0;
}
double Config::region_double(int region, const std::string &key, double dflt) const {
    if (!region_has(region, key)) return dflt;
    const std::string &s = region_extra_[region].at(key);
    char *end = nullptr;
    double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) throw ConfigError("bad numeric value for " + key);
    return v;
}

}  // namespace transfer
