/* Minimal stand-in for the gflags macros used by the reference's host checker
 * sources (the reference's gflags submodule is empty in this checkout).  Only
 * the DEFINE_/DECLARE_ forms are provided: flags become plain globals in the
 * fLx namespaces so the checker sources compile unmodified. This header is
 * part of the oracle build recipe (test infrastructure), not of the product. */
#pragma once
#include <string>
#include <cstdint>
#define SG_SHIM_DEFINE(type, name, val) namespace fLS { type FLAGS_##name = val; } using fLS::FLAGS_##name
#define SG_SHIM_DECLARE(type, name) namespace fLS { extern type FLAGS_##name; } using fLS::FLAGS_##name
#define DEFINE_bool(name, val, txt) SG_SHIM_DEFINE(bool, name, val)
#define DEFINE_int32(name, val, txt) SG_SHIM_DEFINE(int32_t, name, val)
#define DEFINE_uint32(name, val, txt) SG_SHIM_DEFINE(uint32_t, name, val)
#define DEFINE_int64(name, val, txt) SG_SHIM_DEFINE(int64_t, name, val)
#define DEFINE_double(name, val, txt) SG_SHIM_DEFINE(double, name, val)
#define DEFINE_string(name, val, txt) SG_SHIM_DEFINE(std::string, name, val)
#define DECLARE_bool(name) SG_SHIM_DECLARE(bool, name)
#define DECLARE_int32(name) SG_SHIM_DECLARE(int32_t, name)
#define DECLARE_uint32(name) SG_SHIM_DECLARE(uint32_t, name)
#define DECLARE_int64(name) SG_SHIM_DECLARE(int64_t, name)
#define DECLARE_double(name) SG_SHIM_DECLARE(double, name)
#define DECLARE_string(name) SG_SHIM_DECLARE(std::string, name)
