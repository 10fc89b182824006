// Config parser (see config.h).
//
// The keys of radiation.cfg are described by one table (kKeys): the prefix
// that selects the key, the type of its value, whether it belongs to the
// global part of the file or to a [region r] section, and the field that
// receives it.  A line is matched against the prefixes in table order, the
// way the reference selects its branch (Config.cpp:20-112); the value after
// '=' is parsed like the reference's sscanf patterns ("key = %d", "key = %lf":
// blanks optional around '=', leading blanks before the number, anything
// after the number ignored), and a path takes the rest of the line after
// "key = ".  Lines that match no key are kept as additive key/value pairs.
#include "config.h"

#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>

namespace transfer {

namespace {

enum class Kind { Int, Real, Path, Count };
enum class Scope { Global, Region };

// One recognised key.  `field` names the Config member written (see apply()).
struct KeySpec {
    const char *prefix;   // selects the key (prefix match, like strncmp)
    const char *name;     // the key as it appears in messages
    Kind kind;
    Scope scope;
    int field;
};

enum Field { F_KAPPA, F_IP, F_MESH, F_OUT, F_NREG, F_MAXK, F_DEV, F_SOLTYPE, F_DUMP, F_PREC };

// Order matters only where one prefix is a prefix of another line's key
// (none of these are); it follows the reference's branch order.
const KeySpec kKeys[] = {
    {"kappa", "kappa", Kind::Real, Scope::Region, F_KAPPA},
    {"Ip", "Ip", Kind::Real, Scope::Region, F_IP},
    {"meshfile = ", "meshfile", Kind::Path, Scope::Global, F_MESH},
    {"outfile = ", "outfile", Kind::Path, Scope::Global, F_OUT},
    {"numregs", "numregs", Kind::Count, Scope::Global, F_NREG},
    {"angorder", "angorder", Kind::Int, Scope::Global, F_MAXK},
    {"device", "device", Kind::Int, Scope::Global, F_DEV},
    {"soltype", "soltype", Kind::Int, Scope::Global, F_SOLTYPE},
    {"dump", "dump", Kind::Int, Scope::Global, F_DUMP},
    {"precondition", "precondition", Kind::Int, Scope::Global, F_PREC},
};

const long kMaxRegions = 1000000;

std::string trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// After the key's prefix: optional blanks, '=', then the text of the value
// (blanks before it are left for strtod/strtol, which skip them).
const char *after_equals(const char *p) {
    while (*p && std::isspace(static_cast<unsigned char>(*p))) p++;
    return *p == '=' ? p + 1 : nullptr;
}

}  // namespace

Config::Config(const char *cfgfile) {
    FILE *f = std::fopen(cfgfile, "r");
    if (!f) throw ConfigError(std::string("cannot open configuration file ") + cfgfile);
    char buf[1024];
    int line = 0, section = -1;
    auto fail = [&](const std::string &msg) {
        std::fclose(f);
        std::ostringstream os;
        os << cfgfile << ", line " << line << ": " << msg;
        throw ConfigError(os.str());
    };

    // parse the value of `k` from `text` (the line after the prefix) into
    // the field; returns false when the line does not hold a value of the
    // key's type
    auto apply = [&](const KeySpec &k, const char *text) -> bool {
        if (k.kind == Kind::Path) {
            std::string v(text);
            while (!v.empty() && (v.back() == '\n' || v.back() == '\r')) v.pop_back();
            (k.field == F_MESH ? meshfn_ : outfn_) = v;
            return true;
        }
        const char *val = after_equals(text);
        if (!val) return false;
        char *end = nullptr;
        errno = 0;
        if (k.kind == Kind::Real) {
            double x = std::strtod(val, &end);
            if (end == val) return false;
            (k.field == F_KAPPA ? kappa_ : Ip_)[section] = x;
            return true;
        }
        long x = std::strtol(val, &end, 10);
        if (end == val || errno == ERANGE) return false;
        switch (k.field) {
            case F_NREG:
                if (x < 0 || x > kMaxRegions)
                    fail("numregs = " + std::to_string(x) + " is outside 0.." + std::to_string(kMaxRegions));
                nreg_ = static_cast<int>(x);
                kappa_.assign(nreg_ + 1, 0.0);
                Ip_.assign(nreg_ + 1, 0.0);
                region_extra_.assign(nreg_ + 1, std::map<std::string, std::string>());
                break;
            case F_MAXK: maxk_ = static_cast<int>(x); break;
            case F_DEV: dev_ = static_cast<int>(x); break;
            case F_SOLTYPE: soltype_ = static_cast<int>(x); break;
            case F_DUMP: dump_ = static_cast<int>(x); break;
            case F_PREC: prec_ = static_cast<int>(x); break;
        }
        return true;
    };

    while (std::fgets(buf, sizeof buf, f)) {
        line++;
        if (buf[0] == '#' || buf[0] == '\n') continue;
        if (buf[0] == '[') {
            int r = 0;
            if (std::sscanf(buf, "[region %d]", &r) != 1)
                fail("a section header must read [region <number>]");
            if (nreg_ < 0) fail("[region " + std::to_string(r) + "] comes before numregs");
            if (r < 0 || r > nreg_)
                fail("[region " + std::to_string(r) + "] is outside 0..numregs = " + std::to_string(nreg_));
            section = r;
            continue;
        }
        const KeySpec *key = nullptr;
        for (const KeySpec &k : kKeys)
            if (!std::strncmp(buf, k.prefix, std::strlen(k.prefix))) {
                key = &k;
                break;
            }
        if (key) {
            const std::string name(key->name);
            if (key->scope == Scope::Region && section < 0)
                fail("'" + name + "' belongs in a [region r] section");
            if (key->scope == Scope::Global && section >= 0)
                fail("'" + name + "' is a global key but appears in [region " + std::to_string(section) + "]");
            if (!apply(*key, buf + std::strlen(key->prefix)))
                fail("'" + name + "' needs a " + (key->kind == Kind::Real ? "number" : "whole number") +
                     " after '=': " + trim(buf));
            continue;
        }
        // additive "key = value" lines (the reference skips them)
        std::string s(buf);
        size_t eq = s.find('=');
        if (eq == std::string::npos) continue;
        std::string k = trim(s.substr(0, eq)), v = trim(s.substr(eq + 1));
        if (k.empty()) continue;
        if (section >= 0) region_extra_[section][k] = v;
        else extra_[k] = v;
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
    if (end == it->second.c_str()) throw ConfigError("'" + key + "' is not a number: " + it->second);
    return v;
}
int Config::get_int(const std::string &key, int dflt) const {
    auto it = extra_.find(key);
    if (it == extra_.end()) return dflt;
    char *end = nullptr;
    long v = std::strtol(it->second.c_str(), &end, 10);
    if (end == it->second.c_str()) throw ConfigError("'" + key + "' is not a whole number: " + it->second);
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
    if (end == s.c_str())
        throw ConfigError("'" + key + "' of [region " + std::to_string(region) + "] is not a number: " + s);
    return v;
}

}  // namespace transfer
