// Status strings and the per-thread last-error message of the C ABI.
#include <stdarg.h>
#include <stdio.h>

#include <atomic>

#include "common.cuh"

namespace nefct {

static thread_local char g_last_error[512] = "";

// Launch-shape knobs; every value runs the same per-ray arithmetic (the
// forward's output does not depend on them).
static std::atomic<int> g_tune[NEFCT_TUNE_COUNT] = {{8}, {0}, {3}};

static bool tune_valid(int key, int value)
{
    switch (key) {
    case NEFCT_TUNE_CB_ROWS: return value == 1 || value == 2 || value == 4 || value == 8;
    case NEFCT_TUNE_CB_ORDER: return value == 0 || value == 1;
    case NEFCT_TUNE_CB_WALK: return value >= 0 && value <= 3;
    default: return false;
    }
}

int tune_get(int key) { return (key >= 0 && key < NEFCT_TUNE_COUNT) ? g_tune[key].load(std::memory_order_relaxed) : 0; }

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

nefct_status nefct_tune_set(int32_t key, int32_t value)
{
    if (!nefct::tune_valid(key, value)) return nefct::fail(NEFCT_ERR_INVALID, "bad tuning key %d / value %d", key, value);
    nefct::g_tune[key].store(value, std::memory_order_relaxed);
    return NEFCT_OK;
}

int32_t nefct_tune_get(int32_t key) { return nefct::tune_get(key); }

}  // extern "C"
