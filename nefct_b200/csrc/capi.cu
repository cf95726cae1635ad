// Status strings and the per-thread last-error message of the C ABI.
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace nefct {

static thread_local char g_last_error[512] = "";

nefct_status fail(nefct_status st, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return st;
}

nefct_status cuda_fail(cudaError_t e, const char *what)
{
    return fail(NEFCT_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

}  // namespace nefct

extern "C" {

const char *nefct_version(void) { return "nefct_b200 0.1.0 (sm_100a)"; }

const char *nefct_status_string(nefct_status st)
{
    switch (st) {
    case NEFCT_OK: return "ok";
    case NEFCT_ERR_INVALID: return "invalid argument";
    case NEFCT_ERR_CUDA: return "CUDA error";
    case NEFCT_ERR_WORKSPACE: return "workspace missing or too small";
    case NEFCT_ERR_TIMEOUT: return "bounded device wait expired";
    case NEFCT_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
    }
}

const char *nefct_last_error(void) { return nefct::g_last_error; }

}  // extern "C"
