// Cone-beam Siddon kernels (forward and transpose) and their launch
// dispatch, shared by cb_forward.cu and cb_backward.cu, which instantiate
// them (one direction per translation unit), and siddon.cu (host side).
//
// Two walks, chosen per direction by NEFCT_TUNE_CB_WALK:
//  * thread per ray (cb_forward_kernel / cb_backward_kernel): 32 adjacent
//    detector columns x blockDim.y rows per CTA, each warp 32 neighbouring
//    columns of one row; volume x-fastest plus a y-fastest copy for x-driven
//    rays;
//  * column warps (cb_colwarp_kernel, FP32): each warp 32 consecutive rows
//    of one column, blockDim.y columns per CTA, over a z-fastest copy of the
//    volume (colwarp.cuh); the forward's cb_colwarp_rows_kernel gives each
//    lane two rows (l and l + 32) of a 64-row tile.
// The grid runs (column tile, view, row band) with the row band slowest, or
// (column tile, row band, view).  Per-view cos/sin/z-offset ride in the
// kernel parameters.
#pragma once

#include <type_traits>

#include "colwarp.cuh"

namespace nefct {

template <typename T> struct CBParams {
    GridDev<T> g;
    int na, nb, nvc, v0, nv_total;
    RayGeom<T> rg;
    int band_major;
    uint32_t flags;
    const T *vol;        // x-fastest volume (forward source)
    const T *volT;       // y-fastest copy for x-driven rays (thread walk) or z-fastest copy (column warps)
    const T *sino;       // backward source, full sinogram
    T *out;              // forward: full sinogram; backward: x-fastest volume
    T *outT;             // backward: y-fastest or z-fastest accumulator, or nullptr
    unsigned long long *fix, *fixT;   // deterministic backward: integer accumulators
    const float *fix_scale;           // deterministic backward: power-of-two scale (device)
    unsigned long long *count;
    ViewTable<T> tab;
};

template <typename T>
__device__ __forceinline__ void cb_ray(const CBParams<T> &p, int ia, int ib, int iv, T *r)
{
    cb_ray(p.rg, p.tab.cs[iv], p.tab.sn[iv], p.tab.off[iv], ia, ib, r);
}

// Detector cell of this thread (thread walk): 32 columns x blockDim.y rows
// per CTA; grid (column tile, view, row band) when band_major, else (column
// tile, row band, view).
template <typename T>
__device__ __forceinline__ void cb_cell(const CBParams<T> &p, int &ia, int &ib, int &iv)
{
    ia = blockIdx.x * 32 + threadIdx.x;
    if (p.band_major) { iv = blockIdx.y; ib = blockIdx.z * blockDim.y + threadIdx.y; }
    else { ib = blockIdx.y * blockDim.y + threadIdx.y; iv = blockIdx.z; }
}

// Sinogram value of a ray for the transpose; Q8: the reference's cylindrical
// backprojection reads ia + iv*na + ib*na*nb (reads past the end count as 0).
template <typename T> __device__ __forceinline__ T cb_sino_value(const CBParams<T> &p, int ia, int ib, int iv)
{
    const size_t total = (size_t)p.na * p.nb * p.nv_total;
    const size_t vg = (size_t)(p.v0 + iv);
    const size_t id = (p.flags & NEFCT_Q8_INDEX) ? (size_t)ia + vg * p.na + (size_t)ib * p.na * p.nb
                                                 : vg * p.na * p.nb + (size_t)ib * p.na + ia;
    return id < total ? p.sino[id] : (T)0;
}

template <typename T, bool DIV, bool EXACT = false>
__global__ void __launch_bounds__(256) cb_forward_kernel(const __grid_constant__ CBParams<T> p)
{
    int ia, ib, iv;
    cb_cell(p, ia, ib, iv);
    if (ia >= p.na || ib >= p.nb) return;
    T r[6];
    cb_ray(p, ia, ib, iv, r);
    const T acc = ray_forward<T, DIV, EXACT>(p.g, r, p.flags, p.vol, p.volT);
    p.out[(size_t)(p.v0 + iv) * p.na * p.nb + (size_t)ib * p.na + ia] = acc;
}

template <typename T, bool DIV, bool EXACT = false>
__global__ void __launch_bounds__(256) cb_backward_kernel(const __grid_constant__ CBParams<T> p)
{
    int ia, ib, iv;
    cb_cell(p, ia, ib, iv);
    if (ia >= p.na || ib >= p.nb) return;
    const T y = cb_sino_value(p, ia, ib, iv);
    if (y == (T)0) return;
    T r[6];
    cb_ray(p, ia, ib, iv, r);
    ray_backward<T, DIV, EXACT>(p.g, r, p.flags, y, p.out, p.outT);
}

// One lane of a column warp (the whole warp calls it together).  has: the
// lane has a ray r; FWD: gathers from the z-fastest copy volZ into *out;
// otherwise reduces y times the ray's weights into the z-fastest accumulator
// accZ, or (FIX) as 64-bit fixed-point integers (value * weight * scale,
// rounded) into fixZ.  Rays without a contribution (outside the detector,
// missing the grid, zero value) stay in the warp's walk with every slot
// inactive.
template <bool DIV, bool FWD, bool FIX = false>
__device__ __forceinline__ void colwarp_lane(const GridDev<float> &g, const float *r, bool has, uint32_t flags,
                                             const float *__restrict__ volZ, float *out, float y, float *accZ,
                                             unsigned long long *fixZ = nullptr, float scale = 0.f)
{
    Walk<float> w{};
    const bool live = has && (FWD || y != 0.f) && setup_walk(g, r, flags, w);
    if (!__any_sync(0xffffffffu, live)) {
        if (FWD && has) *out = 0.f;
        return;
    }
    ColShared c;
    ColLane L;
    int K0, K1, KI0, KI1;
    if (!col_setup(g, w, live, c, L, K0, K1, KI0, KI1)) {
        // rays of the column disagree on the shared parameters: walk alone
        unsigned su, sv;
        col_strides(g, w.xdrive, su, sv);
        if (FWD) {
            const float v = live ? gather_walk<float, DIV, false, false>(w, g, volZ, (int)su, (int)sv, 1) : 0.f;
            if (has) *out = v;
        } else if (live && FIX) {
            scatter_walk_fixed<float, DIV, false>(w, g, fixZ, (int)su, (int)sv, 1, y, scale);
        } else if (live) {
            scatter_walk<float, DIV, false, false>(w, g, accZ, (int)su, (int)sv, 1, y);
        }
        return;
    }
    if constexpr (FWD) {
        float acc = 0.f;
        // interior slabs load every slot unpredicated: an inactive slot has
        // ratio 0 and a valid index (so a volume holding +-inf may give NaN
        // where the reference gives +-inf); lanes without a ray are discarded
        auto f = [&](const auto &s) {
            float v[s.n];
#pragma unroll
            for (int i = 0; i < s.n; ++i) v[i] = (!s.checked || s.ok[i]) ? __ldg(volZ + s.idx[i]) : 0.f;
#pragma unroll
            for (int i = 0; i < s.n; ++i) acc += v[i] * s.r[i];
        };
        col_walk_any<DIV, 0>(c, L, K0, K1, KI0, KI1, g, f);
        if (has) *out = live ? acc * w.W : 0.f;
    } else if constexpr (FIX) {
        const float yw = y * w.W;
        auto f = [&](const auto &s) {
#pragma unroll
            for (int i = 0; i < s.n; ++i)
                if (s.ok[i]) atomicAdd(fixZ + s.idx[i], (unsigned long long)to_fixed((yw * s.r[i]) * scale));
        };
        col_walk_any<DIV, 1>(c, L, K0, K1, KI0, KI1, g, f);
    } else {
        const float yw = y * w.W;
        auto f = [&](const auto &s) {
            if constexpr (s.n == 2) {
                // the two-slot split's weights are r and 1 - r: y w (1 - r) in one rounding
                if (s.ok[0]) atomicAdd(accZ + s.idx[0], yw * s.r[0]);
                if (s.ok[1]) atomicAdd(accZ + s.idx[1], fmaf(-yw, s.r[0], yw));
            } else {
#pragma unroll
                for (int i = 0; i < s.n; ++i)
                    if (s.ok[i]) atomicAdd(accZ + s.idx[i], yw * s.r[i]);
            }
        };
        col_walk_any<DIV, 2>(c, L, K0, K1, KI0, KI1, g, f);
    }
}

// R rays per lane (rows l, l + 32, ... of the column): the same walk and
// arithmetic per ray as colwarp_lane, with the warp's slab table and split
// decisions shared by all 32 R rays.  Float forward (FWD) and float
// transpose only.
template <bool DIV, bool FWD, int R>
__device__ __forceinline__ void colwarp_rows(const GridDev<float> &g, const float (&r)[R][6], const bool (&has)[R],
                                             uint32_t flags, const float *__restrict__ volZ, float *const (&out)[R],
                                             const float (&y)[R], float *accZ)
{
    Walk<float> w[R];
    bool live[R];
    bool any = false;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        w[k] = Walk<float>{};
        live[k] = has[k] && (FWD || y[k] != 0.f) && setup_walk(g, r[k], flags, w[k]);
        any = any || live[k];
    }
    if (!__any_sync(0xffffffffu, any)) {
        if (FWD) {
#pragma unroll
            for (int k = 0; k < R; ++k)
                if (has[k]) *out[k] = 0.f;
        }
        return;
    }
    ColShared c;
    ColLane L[R];
    int K0, K1, KI0, KI1;
    if (!col_setup_rows<R>(g, w, live, c, L, K0, K1, KI0, KI1)) {
        // rays of the column disagree on the shared parameters: each walks alone
#pragma unroll
        for (int k = 0; k < R; ++k) {
            unsigned su, sv;
            col_strides(g, w[k].xdrive, su, sv);
            if (FWD) {
                const float v = live[k] ? gather_walk<float, DIV, false, false>(w[k], g, volZ, (int)su, (int)sv, 1) : 0.f;
                if (has[k]) *out[k] = v;
            } else if (live[k]) {
                scatter_walk<float, DIV, false, false>(w[k], g, accZ, (int)su, (int)sv, 1, y[k]);
            }
        }
        return;
    }
    if constexpr (FWD) {
        float acc[R];
#pragma unroll
        for (int k = 0; k < R; ++k) acc[k] = 0.f;
        auto f = [&](const auto &s, int k) {
            float v[s.n];
#pragma unroll
            for (int i = 0; i < s.n; ++i) v[i] = (!s.checked || s.ok[i]) ? __ldg(volZ + s.idx[i]) : 0.f;
#pragma unroll
            for (int i = 0; i < s.n; ++i) acc[k] += v[i] * s.r[i];
        };
        col_walk_any_rows<DIV, 0, R>(c, L, K0, K1, KI0, KI1, g, f);
#pragma unroll
        for (int k = 0; k < R; ++k)
            if (has[k]) *out[k] = live[k] ? acc[k] * w[k].W : 0.f;
    } else {
        float yw[R];
#pragma unroll
        for (int k = 0; k < R; ++k) yw[k] = y[k] * w[k].W;
        auto f = [&](const auto &s, int k) {
            if constexpr (s.n == 2) {
                if (s.ok[0]) atomicAdd(accZ + s.idx[0], yw[k] * s.r[0]);
                if (s.ok[1]) atomicAdd(accZ + s.idx[1], fmaf(-yw[k], s.r[0], yw[k]));
            } else {
#pragma unroll
                for (int i = 0; i < s.n; ++i)
                    if (s.ok[i]) atomicAdd(accZ + s.idx[i], yw[k] * s.r[i]);
            }
        };
        col_walk_any_rows<DIV, 2, R>(c, L, K0, K1, KI0, KI1, g, f);
    }
}

// Column warps: warp = rows [32*tile, 32*tile + 32) of column ia at view iv,
// over the z-fastest copy p.volT (forward, into p.out) or accumulator p.outT.
// (at most 64 registers: 4 CTAs of 256 threads per SM; measured faster than
// the unconstrained 70)
template <bool DIV, bool FWD>
__global__ void __launch_bounds__(256, 4) cb_colwarp_kernel(const __grid_constant__ CBParams<float> p)
{
    const int lane = threadIdx.x;
    const int ia = blockIdx.x * blockDim.y + threadIdx.y;
    int ib, iv;
    if (p.band_major) { iv = blockIdx.y; ib = blockIdx.z * 32 + lane; }
    else { ib = blockIdx.y * 32 + lane; iv = blockIdx.z; }
    if (ia >= p.na) return;                       // uniform across the warp
    const bool has = ib < p.nb;
    float y = 0.f;
    if (!FWD && has) y = cb_sino_value(p, ia, ib, iv);
    float r[6];
    cb_ray(p, ia, has ? ib : 0, iv, r);
    float *const out = FWD ? p.out + (size_t)(p.v0 + iv) * p.na * p.nb + (size_t)ib * p.na + ia : nullptr;
    colwarp_lane<DIV, FWD>(p.g, r, has, p.flags, p.volT, out, y, p.outT);
}

// Rays per lane of the float column-warp kernels, per direction.  Measured
// (512^3, 180 of 720 views of 1024 x 768; 256^3, 360 views of 512 x 384):
// two rays per lane take the forward from 79.6 to 77.7 ms and from 19.1 to
// 18.8 ms (80 registers, 3 CTAs of 256 per SM; bit-identical output) but
// the transpose from 97.8 to 100.2 ms, so the transpose keeps one.
#ifndef NEFCT_COL_ROWS_FWD
#define NEFCT_COL_ROWS_FWD 2
#endif
#ifndef NEFCT_COL_ROWS_BWD
#define NEFCT_COL_ROWS_BWD 1
#endif
#ifndef NEFCT_COL_MINB
#define NEFCT_COL_MINB 3
#endif

// Column warps with R rays per lane: warp = rows [32 R tile, 32 R (tile + 1))
// of column ia at view iv (at most 80 registers: 3 CTAs of 256 per SM).
template <bool DIV, bool FWD, int R>
__global__ void __launch_bounds__(256, NEFCT_COL_MINB) cb_colwarp_rows_kernel(const __grid_constant__ CBParams<float> p)
{
    const int lane = threadIdx.x;
    const int ia = blockIdx.x * blockDim.y + threadIdx.y;
    const int tile = p.band_major ? blockIdx.z : blockIdx.y;
    const int iv = p.band_major ? blockIdx.y : blockIdx.z;
    if (ia >= p.na) return;                       // uniform across the warp
    float r[R][6];
    bool has[R];
    float y[R];
    float *out[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int ib = (tile * R + k) * 32 + lane;
        has[k] = ib < p.nb;
        y[k] = (!FWD && has[k]) ? cb_sino_value(p, ia, ib, iv) : 0.f;
        cb_ray(p, ia, has[k] ? ib : 0, iv, r[k]);
        out[k] = FWD ? p.out + (size_t)(p.v0 + iv) * p.na * p.nb + (size_t)ib * p.na + ia : nullptr;
    }
    colwarp_rows<DIV, FWD, R>(p.g, r, has, p.flags, p.volT, out, y, p.outT);
}

// Launch shape of the thread walk for nvc views (see cb_cell).
template <typename T>
static inline void cb_shape(CBParams<T> &p, int na, int nb, int nvc, dim3 &grid, dim3 &block)
{
    const int rows = tune_get(NEFCT_TUNE_CB_ROWS);
    p.band_major = tune_get(NEFCT_TUNE_CB_ORDER) == 0;
    block = dim3(32, rows);
    const unsigned bands = (unsigned)((nb + rows - 1) / rows);
    grid = p.band_major ? dim3((na + 31) / 32, nvc, bands) : dim3((na + 31) / 32, bands, nvc);
}

// Launch shape of the column warps: NEFCT_TUNE_CB_ROWS columns (warps) per
// CTA, 32 rows per warp.
template <typename T>
static inline void cb_colwarp_shape(CBParams<T> &p, int na, int nb, int nvc, dim3 &grid, dim3 &block,
                                    int rays_per_lane = 1)
{
    const int cols = tune_get(NEFCT_TUNE_CB_ROWS);
    p.band_major = tune_get(NEFCT_TUNE_CB_ORDER) == 0;
    block = dim3(32, cols);
    const unsigned tiles = (unsigned)((nb + 32 * rays_per_lane - 1) / (32 * rays_per_lane));
    grid = p.band_major ? dim3((na + cols - 1) / cols, nvc, tiles) : dim3((na + cols - 1) / cols, tiles, nvc);
}

// The walk skips its divisions when both transverse pitches equal the x pitch.
template <typename T> static inline bool cubic(const GridDev<T> &g) { return g.dy == (T)1 && g.dz == (T)1; }

// Column warps apply to FP32 slab walks with a workspace; the z-fastest
// copy's transposes launch ny planes (grid z), and the packed v floors hold
// n + 3 in 16 bits.
template <typename T> static inline bool cb_use_colwarp(const nefct_grid &g, uint32_t flags, bool forward)
{
    return sizeof(T) == sizeof(float) && (tune_get(NEFCT_TUNE_CB_WALK) & (forward ? 1 : 2)) != 0 &&
           !(flags & (NEFCT_EXACT | NEFCT_NO_TRANSPOSE | NEFCT_DETERMINISTIC)) && g.ny <= 65535 &&
           g.nx + 3 < 65536 && g.ny + 3 < 65536;
}

// Launches the thread-walk forward (FWD) or transpose kernel for the views
// set in p.
template <typename T, bool FWD>
static inline cudaError_t cb_launch(CBParams<T> &p, int na, int nb, int nvc, uint32_t flags, cudaStream_t s)
{
    dim3 grid, block;
    cb_shape(p, na, nb, nvc, grid, block);
    const bool exact = (flags & NEFCT_EXACT) != 0, div = !cubic(p.g);
    if constexpr (FWD) {
        if (exact) cb_forward_kernel<T, false, true><<<grid, block, 0, s>>>(p);
        else if (div) cb_forward_kernel<T, true><<<grid, block, 0, s>>>(p);
        else cb_forward_kernel<T, false><<<grid, block, 0, s>>>(p);
    } else {
        if (exact) cb_backward_kernel<T, false, true><<<grid, block, 0, s>>>(p);
        else if (div) cb_backward_kernel<T, true><<<grid, block, 0, s>>>(p);
        else cb_backward_kernel<T, false><<<grid, block, 0, s>>>(p);
    }
    return cudaGetLastError();
}

template <bool FWD>
static inline cudaError_t cb_launch_colwarp(CBParams<float> &p, int na, int nb, int nvc, cudaStream_t s)
{
    dim3 grid, block;
    constexpr int R = FWD ? NEFCT_COL_ROWS_FWD : NEFCT_COL_ROWS_BWD;
    if constexpr (R > 1) {
        cb_colwarp_shape(p, na, nb, nvc, grid, block, R);
        if (cubic(p.g)) cb_colwarp_rows_kernel<false, FWD, R><<<grid, block, 0, s>>>(p);
        else cb_colwarp_rows_kernel<true, FWD, R><<<grid, block, 0, s>>>(p);
    } else {
        cb_colwarp_shape(p, na, nb, nvc, grid, block);
        if (cubic(p.g)) cb_colwarp_kernel<false, FWD><<<grid, block, 0, s>>>(p);
        else cb_colwarp_kernel<true, FWD><<<grid, block, 0, s>>>(p);
    }
    return cudaGetLastError();
}

// Launches the forward / transpose kernels for the views set in p: the
// thread walk, or the column warps when colwarp (p.volT / p.outT then hold
// the z-fastest copy / accumulator).  Defined in cb_forward.cu /
// cb_backward.cu for float and double.
template <typename T>
cudaError_t cb_launch_forward(CBParams<T> &p, int na, int nb, int nvc, uint32_t flags, cudaStream_t s,
                              bool colwarp = false);
template <typename T>
cudaError_t cb_launch_backward(CBParams<T> &p, int na, int nb, int nvc, uint32_t flags, cudaStream_t s,
                               bool colwarp = false);

}  // namespace nefct
