// Command-line flags for the hybrid_* samples, compatible with the subset of
// gflags the reference samples use (the reference's gflags submodule is empty,
// .gitmodules:4-6): DEFINE_/DECLARE_ bool/int32/double/string, parsing of
// --name=value, --name value, -name, --name / --noname for booleans, --help,
// and FlagSaver for the interactive / command-file sessions
// (include/utils/app_skeleton.h:116-139).  Unknown flags are an error, as in
// gflags.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace sgflags {

enum Kind { BOOL, INT32, DOUBLE, STRING };

struct Flag {
    std::string name;
    Kind kind;
    void *ptr;
    std::string help;
};

inline std::vector<Flag> &registry() {
    static std::vector<Flag> r;
    return r;
}

struct Registrar {
    Registrar(const char *name, Kind k, void *p, const char *help) { registry().push_back({name, k, p, help}); }
};

inline Flag *find(const std::string &n) {
    for (auto &f : registry())
        if (f.name == n) return &f;
    return nullptr;
}

inline bool set_value(Flag &f, const std::string &v) {
    char *end = nullptr;
    switch (f.kind) {
        case BOOL:
            if (v == "true" || v == "1" || v == "yes" || v.empty()) *(bool *)f.ptr = true;
            else if (v == "false" || v == "0" || v == "no") *(bool *)f.ptr = false;
            else return false;
            return true;
        case INT32: {
            long x = std::strtol(v.c_str(), &end, 10);
            if (!end || *end || v.empty()) return false;
            *(int32_t *)f.ptr = (int32_t)x;
            return true;
        }
        case DOUBLE: {
            double x = std::strtod(v.c_str(), &end);
            if (!end || *end || v.empty()) return false;
            *(double *)f.ptr = x;
            return true;
        }
        case STRING:
            *(std::string *)f.ptr = v;
            return true;
    }
    return false;
}

inline void usage(const char *prog) {
    std::printf("usage: %s [flags]\n", prog);
    for (auto &f : registry()) std::printf("  --%s  %s\n", f.name.c_str(), f.help.c_str());
}

// Parses flags, leaving positional arguments in argv.  Returns false on an
// unknown flag or a malformed value (message on stderr).
inline bool ParseCommandLineFlags(int *argc, char ***argv, bool remove_flags = true) {
    std::vector<char *> rest;
    rest.push_back((*argv)[0]);
    for (int i = 1; i < *argc; ++i) {
        std::string a = (*argv)[i];
        if (a.size() < 2 || a[0] != '-') {
            rest.push_back((*argv)[i]);
            continue;
        }
        std::string body = a.substr(a[1] == '-' ? 2 : 1);
        if (body == "help") {
            usage((*argv)[0]);
            std::exit(0);
        }
        std::string name = body, val;
        bool has_val = false;
        const size_t eq = body.find('=');
        if (eq != std::string::npos) {
            name = body.substr(0, eq);
            val = body.substr(eq + 1);
            has_val = true;
        }
        Flag *f = find(name);
        if (!f && name.rfind("no", 0) == 0 && !has_val) {
            Flag *g = find(name.substr(2));
            if (g && g->kind == BOOL) {
                *(bool *)g->ptr = false;
                continue;
            }
        }
        if (!f) {
            std::fprintf(stderr, "ERROR: unknown command line flag '%s'\n", name.c_str());
            return false;
        }
        if (!has_val && f->kind != BOOL) {
            if (i + 1 >= *argc) {
                std::fprintf(stderr, "ERROR: flag '%s' is missing its argument\n", name.c_str());
                return false;
            }
            val = (*argv)[++i];
            has_val = true;
        }
        if (!set_value(*f, val)) {
            std::fprintf(stderr, "ERROR: illegal value '%s' specified for flag '%s'\n", val.c_str(), name.c_str());
            return false;
        }
    }
    if (remove_flags) {
        for (size_t k = 0; k < rest.size(); ++k) (*argv)[k] = rest[k];
        *argc = (int)rest.size();
    }
    return true;
}

// Saves every flag value and restores it on destruction.
class FlagSaver {
    std::vector<std::string> s_;
    std::vector<double> d_;
    std::vector<int32_t> i_;
    std::vector<char> b_;

   public:
    FlagSaver() {
        for (auto &f : registry()) {
            s_.push_back(f.kind == STRING ? *(std::string *)f.ptr : std::string());
            d_.push_back(f.kind == DOUBLE ? *(double *)f.ptr : 0.0);
            i_.push_back(f.kind == INT32 ? *(int32_t *)f.ptr : 0);
            b_.push_back(f.kind == BOOL ? *(bool *)f.ptr : 0);
        }
    }
    ~FlagSaver() {
        size_t k = 0;
        for (auto &f : registry()) {
            switch (f.kind) {
                case STRING: *(std::string *)f.ptr = s_[k]; break;
                case DOUBLE: *(double *)f.ptr = d_[k]; break;
                case INT32: *(int32_t *)f.ptr = i_[k]; break;
                case BOOL: *(bool *)f.ptr = b_[k]; break;
            }
            ++k;
        }
    }
};

}  // namespace sgflags

#define SGF_DEFINE(type, kind, name, val, txt) \
    type FLAGS_##name = val;                    \
    static sgflags::Registrar sgf_reg_##name(#name, sgflags::kind, &FLAGS_##name, txt)
#define DEFINE_bool(name, val, txt) SGF_DEFINE(bool, BOOL, name, val, txt)
#define DEFINE_int32(name, val, txt) SGF_DEFINE(int32_t, INT32, name, val, txt)
#define DEFINE_double(name, val, txt) SGF_DEFINE(double, DOUBLE, name, val, txt)
#define DEFINE_string(name, val, txt) SGF_DEFINE(std::string, STRING, name, val, txt)
#define DECLARE_bool(name) extern bool FLAGS_##name
#define DECLARE_int32(name) extern int32_t FLAGS_##name
#define DECLARE_double(name) extern double FLAGS_##name
#define DECLARE_string(name) extern std::string FLAGS_##name
