/* Minimal stand-in for the gflags API used by the reference's host checker
 * sources and its graph converter (the reference's gflags submodule is empty in
 * this checkout).  DEFINE_ forms make plain globals in the fLS namespace and
 * register them, so ParseCommandLineFlags can set them from
 * --name=value / --name value / --name / --noname arguments.  This header is
 * part of the oracle build recipe (test infrastructure), not of the product. */
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace sg_shim {
struct Flag {
    const char *name;
    char type; /* b i u l d s */
    void *ptr;
};
inline std::vector<Flag> &registry() {
    static std::vector<Flag> r;
    return r;
}
struct Reg {
    Reg(const char *n, char t, void *p) { registry().push_back(Flag{n, t, p}); }
};
inline bool set(const Flag &f, const char *v) {
    switch (f.type) {
        case 'b': *(bool *)f.ptr = !(std::strcmp(v, "false") == 0 || std::strcmp(v, "0") == 0); return true;
        case 'i': *(int32_t *)f.ptr = (int32_t)std::strtol(v, nullptr, 10); return true;
        case 'u': *(uint32_t *)f.ptr = (uint32_t)std::strtoul(v, nullptr, 10); return true;
        case 'l': *(int64_t *)f.ptr = (int64_t)std::strtoll(v, nullptr, 10); return true;
        case 'd': *(double *)f.ptr = std::strtod(v, nullptr); return true;
        case 's': *(std::string *)f.ptr = v; return true;
    }
    return false;
}
inline const Flag *find(const std::string &n) {
    for (const Flag &f : registry())
        if (n == f.name) return &f;
    return nullptr;
}
}  // namespace sg_shim

#define SG_SHIM_DEFINE(type, tc, name, val)                       \
    namespace fLS {                                               \
    type FLAGS_##name = val;                                      \
    static sg_shim::Reg sg_shim_reg_##name(#name, tc, &FLAGS_##name); \
    }                                                             \
    using fLS::FLAGS_##name
#define SG_SHIM_DECLARE(type, name) namespace fLS { extern type FLAGS_##name; } using fLS::FLAGS_##name
#define DEFINE_bool(name, val, txt) SG_SHIM_DEFINE(bool, 'b', name, val)
#define DEFINE_int32(name, val, txt) SG_SHIM_DEFINE(int32_t, 'i', name, val)
#define DEFINE_uint32(name, val, txt) SG_SHIM_DEFINE(uint32_t, 'u', name, val)
#define DEFINE_int64(name, val, txt) SG_SHIM_DEFINE(int64_t, 'l', name, val)
#define DEFINE_double(name, val, txt) SG_SHIM_DEFINE(double, 'd', name, val)
#define DEFINE_string(name, val, txt) SG_SHIM_DEFINE(std::string, 's', name, val)
#define DECLARE_bool(name) SG_SHIM_DECLARE(bool, name)
#define DECLARE_int32(name) SG_SHIM_DECLARE(int32_t, name)
#define DECLARE_uint32(name) SG_SHIM_DECLARE(uint32_t, name)
#define DECLARE_int64(name) SG_SHIM_DECLARE(int64_t, name)
#define DECLARE_double(name) SG_SHIM_DECLARE(double, name)
#define DECLARE_string(name) SG_SHIM_DECLARE(std::string, name)

namespace gflags {
/* Sets registered flags from argv; an unknown flag is an error (exit 1).
 * Parsed arguments are removed when remove_flags is true. */
inline void ParseCommandLineFlags(int *argc, char ***argv, bool remove_flags) {
    std::vector<char *> rest;
    rest.push_back((*argv)[0]);
    for (int i = 1; i < *argc; ++i) {
        char *a = (*argv)[i];
        if (a[0] != '-') {
            rest.push_back(a);
            continue;
        }
        std::string s = a + (a[1] == '-' ? 2 : 1);
        std::string name = s, val;
        bool has_val = false;
        const size_t eq = s.find('=');
        if (eq != std::string::npos) {
            name = s.substr(0, eq);
            val = s.substr(eq + 1);
            has_val = true;
        }
        const sg_shim::Flag *f = sg_shim::find(name);
        if (!f && !has_val && name.compare(0, 2, "no") == 0) {
            f = sg_shim::find(name.substr(2));
            if (f && f->type == 'b') {
                *(bool *)f->ptr = false;
                continue;
            }
            f = nullptr;
        }
        if (!f) {
            std::fprintf(stderr, "unknown flag --%s\n", name.c_str());
            std::exit(1);
        }
        if (!has_val) {
            if (f->type == 'b') val = "true";
            else if (i + 1 < *argc) val = (*argv)[++i];
            else {
                std::fprintf(stderr, "flag --%s needs a value\n", name.c_str());
                std::exit(1);
            }
        }
        sg_shim::set(*f, val.c_str());
    }
    if (remove_flags) {
        for (size_t k = 0; k < rest.size(); ++k) (*argv)[k] = rest[k];
        *argc = (int)rest.size();
    }
}
}  // namespace gflags
