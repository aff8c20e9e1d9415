// Run-config front-end: the TOML keys the sample main and HiDEMLib::setup read
// (HiDEM/MeshBlock/MainMeshBlock.cpp:69-102, HiDEMLib/HiDEMLib.h:714-750,
// HiDEMLib/HiDEMGeometry.cpp:82-133) with the reference's command-line overrides
// `--section.key=value` / `--section.key value` / bare `--section.key` = true
// (PLiB/Util/ArgParser.h:170-270). Missing keys keep the MeshBlock defaults.
//
// The parser reads the TOML subset these files use: [table] headers, [[array]] headers
// (their keys are skipped), `key = value` with numbers, booleans, quoted strings and
// (possibly multi-line) arrays of numbers, and # comments.
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "hidem_b200.h"

namespace hidem {
extern thread_local std::string g_nocontext_error;
}

namespace {

std::string trim(const std::string &s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

// strips a # comment that is not inside a quoted string
std::string strip_comment(const std::string &s) {
    bool inStr = false;
    char q = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        char c = s[i];
        if (inStr) {
            if (c == '\\' && q == '"') {
                ++i;
                continue;
            }
            if (c == q) inStr = false;
        } else if (c == '"' || c == '\'') {
            inStr = true;
            q = c;
        } else if (c == '#') {
            return s.substr(0, i);
        }
    }
    return s;
}

int bracket_balance(const std::string &s) {
    int b = 0;
    bool inStr = false;
    char q = 0;
    for (char c : s) {
        if (inStr) {
            if (c == q) inStr = false;
        } else if (c == '"' || c == '\'') {
            inStr = true;
            q = c;
        } else if (c == '[') {
            ++b;
        } else if (c == ']') {
            --b;
        }
    }
    return b;
}

bool parse_toml(const std::string &path, std::map<std::string, std::string> &kv, std::string &err) {
    std::ifstream f(path);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    std::string line, table;
    bool skipping = false;  // inside an [[array of tables]]
    int lineNo = 0;
    while (std::getline(f, line)) {
        ++lineNo;
        std::string s = trim(strip_comment(line));
        if (s.empty()) continue;
        if (s.rfind("[[", 0) == 0) {
            skipping = true;
            continue;
        }
        if (s[0] == '[') {
            size_t e = s.find(']');
            if (e == std::string::npos) {
                err = path + ":" + std::to_string(lineNo) + ": bad table header";
                return false;
            }
            table = trim(s.substr(1, e - 1));
            skipping = false;
            continue;
        }
        size_t eq = s.find('=');
        if (eq == std::string::npos) {
            err = path + ":" + std::to_string(lineNo) + ": expected key = value";
            return false;
        }
        std::string key = trim(s.substr(0, eq));
        std::string val = trim(s.substr(eq + 1));
        while (bracket_balance(val) > 0 && std::getline(f, line)) {
            ++lineNo;
            val += " " + trim(strip_comment(line));
        }
        if (skipping) continue;
        if (key.size() >= 2 && key.front() == '"' && key.back() == '"') key = key.substr(1, key.size() - 2);
        kv[table.empty() ? key : table + "." + key] = val;
    }
    return true;
}

bool as_double(const std::string &v, double &out) {
    std::string s;
    for (char c : v)
        if (c != '_') s += c;
    if (s == "true") { out = 1; return true; }
    if (s == "false") { out = 0; return true; }
    if (s == "inf" || s == "+inf") { out = INFINITY; return true; }
    if (s == "-inf") { out = -INFINITY; return true; }
    char *end = nullptr;
    out = std::strtod(s.c_str(), &end);
    return end && *end == '\0' && !s.empty();
}

bool as_bool(const std::string &v, int32_t &out) {
    if (v == "true" || v == "1") { out = 1; return true; }
    if (v == "false" || v == "0") { out = 0; return true; }
    return false;
}

bool as_triple(const std::string &v, double out[3]) {
    std::string s = trim(v);
    if (s.size() < 2 || s.front() != '[' || s.back() != ']') return false;
    std::stringstream ss(s.substr(1, s.size() - 2));
    std::string item;
    int k = 0;
    while (std::getline(ss, item, ',')) {
        item = trim(item);
        if (item.empty()) continue;
        if (k >= 3 || !as_double(item, out[k])) return false;
        ++k;
    }
    return k == 3;
}

std::string unquote(const std::string &v) {
    if (v.size() >= 2 && (v.front() == '"' || v.front() == '\'') && v.back() == v.front())
        return v.substr(1, v.size() - 2);
    return v;
}

}  // namespace

extern "C" hidem_status hidem_params_from_toml(const char *path, int32_t argc,
                                               const char *const *argv, hidem_params *out,
                                               int64_t *time_steps) {
    hidem::g_nocontext_error.clear();
    if (!out) {
        hidem::g_nocontext_error = "out is NULL";
        return HIDEM_ERR_ARG;
    }
    std::map<std::string, std::string> kv;
    std::string err;
    if (path && *path && !parse_toml(path, kv, err)) {
        hidem::g_nocontext_error = err;
        return HIDEM_ERR_IO;
    }
    // command-line overrides win over the file (ArgParser::getArg)
    for (int i = 0; argv && i < argc; ++i) {
        if (!argv[i]) continue;
        std::string a = argv[i];
        if (a.rfind("-", 0) != 0) continue;
        while (!a.empty() && a[0] == '-') a.erase(0, 1);
        std::string key = a, val = "true";
        size_t eq = a.find('=');
        if (eq != std::string::npos) {
            key = a.substr(0, eq);
            val = a.substr(eq + 1);
        } else if (i + 1 < argc && argv[i + 1] && argv[i + 1][0] != '-') {
            val = argv[++i];
        }
        kv[key] = trim(val);
    }

    hidem_params p;
    hidem_params_default(&p);
    struct NumKey { const char *key; double *dst; };
    const NumKey nums[] = {
        {"general.dt", &p.dt}, {"general.scale", &p.scale}, {"general.E", &p.E},
        {"general.beamWidth", &p.beamWidth}, {"general.damping", &p.damping},
        {"general.dampingRotation", &p.dampingRotation},
        {"general.attractDistance", &p.attractDistance},
        {"general.attractScaleForce", &p.attractScaleForce}, {"general.maxLoad", &p.maxLoad},
        {"general.bendBreak", &p.bendBreak}, {"general.breakTime", &p.breakTime},
        {"general.g", &p.g}, {"general.rhoIce", &p.rhoIce}, {"general.rhoWater", &p.rhoWater},
        {"general.waterLevel", &p.waterLevel}, {"general.airDrag", &p.airDrag},
        {"general.waterDrag", &p.waterDrag}, {"general.bedDrag", &p.bedDrag},
        {"general.bedStiffness", &p.bedStiffness}, {"general.bedInteract", &p.bedInteract},
        {"general.maxVel", &p.maxVel}, {"general.maxRot", &p.maxRot},
        {"general.bedHeight", &p.bedHeight}, {"general.bedFriction", &p.bedFriction},
        {"grid.searchDistanceScale", &p.searchDistanceScale},
    };
    for (const NumKey &k : nums) {
        auto it = kv.find(k.key);
        if (it == kv.end()) continue;
        if (!as_double(it->second, *k.dst)) {
            hidem::g_nocontext_error = std::string(k.key) + ": not a number: " + it->second;
            return HIDEM_ERR_IO;
        }
    }
    struct IntKey { const char *key; int32_t *dst; bool boolean; };
    const IntKey ints[] = {
        {"grid.gridRegenInterval", &p.gridRegenInterval, false},
        {"distribution.firstBalanceTimestep", &p.firstBalanceTimestep, false},
        {"general.xBoundaryMin", &p.boundaryMin[0], true}, {"general.yBoundaryMin", &p.boundaryMin[1], true},
        {"general.zBoundaryMin", &p.boundaryMin[2], true}, {"general.xBoundaryMax", &p.boundaryMax[0], true},
        {"general.yBoundaryMax", &p.boundaryMax[1], true}, {"general.zBoundaryMax", &p.boundaryMax[2], true},
        {"general.useBed", &p.useBed, true}, {"general.useVelocityLimit", &p.useVelocityLimit, true},
        {"general.useBoundary", &p.useBoundary, true}, {"general.useFixed", &p.useFixed, true},
        {"general.useFrontPressure", &p.useFrontPressure, true},
    };
    for (const IntKey &k : ints) {
        auto it = kv.find(k.key);
        if (it == kv.end()) continue;
        double d = 0;
        bool ok = k.boolean ? as_bool(it->second, *k.dst) : as_double(it->second, d);
        if (ok && !k.boolean) *k.dst = (int32_t)d;
        if (!ok) {
            hidem::g_nocontext_error = std::string(k.key) + ": bad value: " + it->second;
            return HIDEM_ERR_IO;
        }
    }
    double tri[3];
    auto lo = kv.find("general.lowerLimit");
    if (lo != kv.end()) {
        if (!as_triple(lo->second, tri)) {
            hidem::g_nocontext_error = "general.lowerLimit: need [x, y, z]";
            return HIDEM_ERR_IO;
        }
        for (int k = 0; k < 3; ++k) p.lowerLimit[k] = tri[k];
    }
    auto hi = kv.find("general.upperLimit");
    if (hi != kv.end()) {
        if (!as_triple(hi->second, tri)) {
            hidem::g_nocontext_error = "general.upperLimit: need [x, y, z]";
            return HIDEM_ERR_IO;
        }
        for (int k = 0; k < 3; ++k) p.upperLimit[k] = tri[k];
    }
    auto pr = kv.find("general.precision");
    if (pr != kv.end()) {
        std::string v = unquote(pr->second);
        if (v == "mixed") p.precision = HIDEM_PREC_MIXED;
        else if (v == "fp64") p.precision = HIDEM_PREC_FP64;
        else {
            hidem::g_nocontext_error = "general.precision: \"mixed\" or \"fp64\"";
            return HIDEM_ERR_IO;
        }
    }
    // geometry.maxRadius = lattice.particleRadius * scale (HiDEMGeometry.cpp:88-92)
    auto rad = kv.find("lattice.particleRadius");
    if (rad != kv.end()) {
        double r = 0;
        if (!as_double(rad->second, r)) {
            hidem::g_nocontext_error = "lattice.particleRadius: not a number";
            return HIDEM_ERR_IO;
        }
        p.maxRadius = r * p.scale;
    }
    if (time_steps) {
        *time_steps = 10000;  // iteration.timeSteps default (HiDEMLib.h:714)
        auto ts = kv.find("iteration.timeSteps");
        double d;
        if (ts != kv.end() && as_double(ts->second, d)) *time_steps = (int64_t)d;
    }
    *out = p;
    return HIDEM_OK;
}
