// Shared definitions of the nefct_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "nefct_b200.h"

namespace nefct {

// Process-wide launch tuning (nefct_tune_set / nefct_tune_get).
int tune_get(int key);

// Records a message for nefct_last_error() and returns the status.
nefct_status fail(nefct_status st, const char *fmt, ...);
// Maps a CUDA error to NEFCT_ERR_CUDA with the call site in the message.
nefct_status cuda_fail(cudaError_t e, const char *what);

#define NEFCT_CHECK_CUDA(call)                                   \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return ::nefct::cuda_fail(e_, #call); \
    } while (0)

#define NEFCT_CHECK_LAUNCH(name)                                 \
    do {                                                         \
        cudaError_t e_ = cudaGetLastError();                     \
        if (e_ != cudaSuccess) return ::nefct::cuda_fail(e_, name); \
    } while (0)

// Approximate reciprocal (PTX rcp.approx.ftz.f32, relative error <= 2^-23).
__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Arithmetic with explicit round-to-nearest so the compiler cannot contract
// a*b+c into one fused operation where the reference's evaluation order has
// two roundings.  Used for every quantity that feeds a floor() or a branch.
template <typename T> struct FP;
template <> struct FP<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
    static __device__ __forceinline__ int ifloor(float a) { return __float2int_rd(a); }
    // ratio of a crossing: a times the approximate reciprocal of b (<= 2 ulp)
    static __device__ __forceinline__ float ratio(float a, float b) { return __fmul_rn(a, rcp_approx(b)); }
    static __device__ __forceinline__ float min(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float max(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float abs(float a) { return fabsf(a); }
};
template <> struct FP<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
    static __device__ __forceinline__ int ifloor(double a) { return __double2int_rd(a); }
    static __device__ __forceinline__ double ratio(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double min(double a, double b) { return fmin(a, b); }
    static __device__ __forceinline__ double max(double a, double b) { return fmax(a, b); }
    static __device__ __forceinline__ double abs(double a) { return fabs(a); }
};

// Pairs of values updated by the same operation sequence (the two
// transverse plane positions).  Each component is rounded by its own scalar
// _rn operation: a paired multiply followed by a paired add may be fused into
// one paired fused multiply-add, which rounds once where the reference
// rounds twice.
template <typename T> struct Pair;
template <> struct Pair<float> {
    float2 v;
    static __device__ __forceinline__ Pair make(float a, float b) { Pair p; p.v = make_float2(a, b); return p; }
    __device__ __forceinline__ float x() const { return v.x; }
    __device__ __forceinline__ float y() const { return v.y; }
    static __device__ __forceinline__ Pair add(Pair a, Pair b) { return make(__fadd_rn(a.v.x, b.v.x), __fadd_rn(a.v.y, b.v.y)); }
    static __device__ __forceinline__ Pair mul(Pair a, Pair b) { return make(__fmul_rn(a.v.x, b.v.x), __fmul_rn(a.v.y, b.v.y)); }
};
template <> struct Pair<double> {
    double a_, b_;
    static __device__ __forceinline__ Pair make(double a, double b) { Pair p; p.a_ = a; p.b_ = b; return p; }
    __device__ __forceinline__ double x() const { return a_; }
    __device__ __forceinline__ double y() const { return b_; }
    static __device__ __forceinline__ Pair add(Pair a, Pair b) { return make(__dadd_rn(a.a_, b.a_), __dadd_rn(a.b_, b.b_)); }
    static __device__ __forceinline__ Pair mul(Pair a, Pair b) { return make(__dmul_rn(a.a_, b.a_), __dmul_rn(a.b_, b.b_)); }
};

// Views handled by one launch; the per-view table travels in the kernel's
// parameter space (broadcast through the constant bank), so no device
// buffer or host->device copy is needed for it.
template <typename T> struct ViewTable {
    static constexpr int kMax = sizeof(T) == 4 ? 1024 : 512;
    T cs[kMax];
    T sn[kMax];
    T off[kMax];
};

}  // namespace nefct
