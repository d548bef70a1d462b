// common.h -- shared host-side helpers for libexcent_b200: status codes, the
// thread-local last-error string, and CUDA call checking that returns a status
// instead of exiting (the reference aborts the process on any CUDA error,
// src/excent.cu:16-17).
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "excent_b200.h"

namespace excent {

typedef unsigned long long ull;

void set_error(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
const char* get_error();

struct Status {
    int code = EXCENT_OK;
    bool ok() const { return code == EXCENT_OK; }
};

}  // namespace excent

// Record a formatted error and return the code from the enclosing function.
#define EX_FAIL(code, ...) do { ::excent::set_error(__VA_ARGS__); return (code); } while (0)
#define EX_CHECK_ARG(cond, ...) do { if (!(cond)) EX_FAIL(EXCENT_ERR_ARG, __VA_ARGS__); } while (0)
#define EX_TRY(expr) do { int rc_ = (expr); if (rc_ != EXCENT_OK) return rc_; } while (0)

#ifdef __CUDACC__
#define EX_CUDA(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
    ::excent::set_error("CUDA error %s (%s) at %s:%d", cudaGetErrorName(e_), cudaGetErrorString(e_), __FILE__, __LINE__); \
    return EXCENT_ERR_CUDA; } } while (0)
#endif
