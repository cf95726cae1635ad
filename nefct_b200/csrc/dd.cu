// Distance-driven FDK backprojection on sm_100a (the detector-driven
// back_project_fdk_kernel of nefct/cc/distance_3d/dist_3d_back_fdk.cu.cc:17-255)
// and its C-ABI entry points (declared in include/nefct_b200.h).
//
// Semantics, per detector bin (ia, ib, iv), in the reference's order of
// operations (explicit round-to-nearest, no contraction):
//  * the bin centre ((i + 0.5) * d + offset - n * d / 2, evaluated in double
//    and rounded, :45-60) and the source give x21, y21, z21; the driving axis
//    is x when |x21| > |y21| (:66);
//  * for every slab of the driving axis the transverse footprint is the span
//    of the four rays through the bin's left/right edges with their x and y
//    components paired both ways (:72-123, :173-223), the z footprint the
//    span of the bin's lower/upper z edges (:125-139);
//  * every voxel inside both footprints gets value * (overlap fraction in v)
//    * (overlap fraction in z) / |u21| * |p2 - p1| * SAD^2 / (SAD + x cos +
//    y sin)^2 (:141-154).  The footprints are evaluated with the reference's
//    operations; the weights divide by multiplying with approximate
//    reciprocals and group the per-column factors (a few ulp per weight).
//
// GPU structure (not the reference's): one warp walks 32 consecutive rows of
// one detector column at one view.  The x and y parts of those rays are
// identical (the bin's x and y do not depend on the row), so the driving axis,
// every slab's transverse footprint and overlap fractions and the FDK weight
// are uniform across the warp; each lane adds its own z footprint.  The
// reductions go to a z-fastest accumulator [y][x][z], where the 32 rows of a
// warp land on neighbouring z of one (x, y) column, so a warp's reduction
// touches one or two 32-byte sectors; one tiled transpose folds it into the
// x-fastest volume.  Per-view cos/sin/offset ride in the kernel parameters.
#include <math.h>
#include <algorithm>

#include "common.cuh"

namespace nefct {

nefct_status zfold(const float *acc, float *vol, const nefct_grid &g, cudaStream_t s);
nefct_status zmajor_copy(const float *in, float *out, const nefct_grid &g, cudaStream_t s);

template <typename T> struct DDParams {
    int nx, ny, nz, na, nb, nvc, v0, cyl, fdk;
    T sid, sad;                   // source-detector, source-axis (the reference's SID, SAD)
    T da, ai, db, bi;
    const T *src;                 // backward: bins [nv][nb][na] (full); forward: the volume
    T *dst;                       // backward: accumulator; forward: bins [nv][nb][na] (full)
    unsigned long long sx, sy, sz;  // volume strides of (ix, iy, iz): z-fastest copy (float) or x-fastest (double)
    ViewTable<T> tab;
};

// (i + 0.5) * d + o - n * d / 2 with the reference's promotions: the first
// part in double, n * d / 2 in float (:45-60); all double in the FP64 build
__device__ __forceinline__ float dd_center(int i, float d, float o, int n)
{
    const float half = __fdiv_rn(__fmul_rn((float)n, d), 2.f);
    return (float)__dsub_rn(__dadd_rn(__dmul_rn((double)i + 0.5, (double)d), (double)o), (double)half);
}
__device__ __forceinline__ double dd_center(int i, double d, double o, int n)
{
    return __dsub_rn(__dadd_rn(__dmul_rn((double)i + 0.5, d), o), __dmul_rn((double)n, d) * 0.5);
}

// i * d + o - n * d / 2 (:78-80)
template <typename T> __device__ __forceinline__ T dd_edge(int i, T d, T o, int n)
{
    return FP<T>::sub(FP<T>::add(FP<T>::mul((T)i, d), o), FP<T>::div(FP<T>::mul((T)n, d), (T)2));
}

// cos/sin of a detector angle: the double-precision functions (rounded for float)
template <typename T> __device__ __forceinline__ void dd_trig(T a, T &c, T &s)
{
    double sd, cd;
    sincos((double)a, &sd, &cd);
    c = (T)cd;
    s = (T)sd;
}

// detector point (x20, y20) of lateral coordinate a (flat: a is the offset
// along the detector; cylindrical: the angle)
template <typename T> __device__ __forceinline__ void dd_det(const DDParams<T> &p, T a, T &x20, T &y20)
{
    if (p.cyl) {
        T c, s;
        dd_trig(a, c, s);
        x20 = FP<T>::sub(FP<T>::mul(p.sid, c), p.sad);
        y20 = FP<T>::mul(p.sid, s);
    } else {
        x20 = FP<T>::sub(p.sid, p.sad);
        y20 = a;
    }
}

template <typename T> __device__ __forceinline__ T dd_min(T a, T b) { return a < b ? a : b; }
template <typename T> __device__ __forceinline__ T dd_max(T a, T b) { return a > b ? a : b; }
template <typename T> __device__ __forceinline__ T dd_abs(T a) { return a > (T)0 ? a : -a; }
// reciprocal for the weight divisions: approximate in float (<= 1 ulp), exact in double
__device__ __forceinline__ float dd_rcp(float x) { return rcp_approx(x); }
__device__ __forceinline__ double dd_rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ int dd_floor(float x) { return (int)floorf(x); }
__device__ __forceinline__ int dd_floor(double x) { return (int)floor(x); }

// One warp walks 32 * R rows (bins) of one detector column at one view (lane
// l takes rows l, l + 32, ...) over the slabs of the column's driving axis.
// FWD false: each lane reduces value * weight into the voxels of its bins'
// footprints (the reference's kernel); FWD true: each lane sums voxel *
// weight over the same voxels with the same weights (the exact transpose)
// into its bins.  With p.fdk false the weight lacks the FDK factor SAD^2 /
// (SAD + x cos + y sin)^2.  The transverse footprint and the FDK factor do
// not depend on the row: the warp evaluates them once per slab and voxel for
// all its 32 * R rows; each row's own arithmetic is unchanged (the forward's
// bits too).  Measured, 256^3, 72 views of 512 x 384, backprojection: 1 / 2
// / 3 / 4 rows per lane 19.7 / 14.2 / 12.7 / 12.4 ms (56 / 54-64 / 64-71 /
// 72-80 registers).
#ifndef NEFCT_DD_ROWS
#define NEFCT_DD_ROWS 4
#endif
static constexpr int kDDRows = NEFCT_DD_ROWS;

template <typename T, bool FWD, int R>
__global__ void __launch_bounds__(128) dd_kernel(const __grid_constant__ DDParams<T> p)
{
    using F = FP<T>;
    constexpr bool kF32 = sizeof(T) == sizeof(float);
    const int lane = threadIdx.x;
    const int ia = blockIdx.x * blockDim.y + threadIdx.y;
    const int iv = blockIdx.z;
    if (ia >= p.na) return;                       // uniform across the warp
    bool has[R], live[R];
    size_t bin[R];
    T value[R];
    bool any = false;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int ib = (blockIdx.y * R + r) * 32 + lane;
        has[r] = ib < p.nb;
        bin[r] = ((size_t)(p.v0 + iv) * p.nb + (has[r] ? ib : 0)) * p.na + ia;
        value[r] = (!FWD && has[r]) ? p.src[bin[r]] : (T)0;
        live[r] = FWD ? has[r] : value[r] != (T)0;
        any = any || live[r];
    }
    if (!FWD && !__any_sync(0xffffffffu, any)) return;

    const T cphi = p.tab.cs[iv], sphi = p.tab.sn[iv], off = p.tab.off[iv];
    const T x1 = F::mul(-p.sad, cphi), y1 = F::mul(-p.sad, sphi), z1 = off;
    T x20, y20;
    dd_det(p, dd_center(ia, p.da, p.ai, p.na), x20, y20);
    const T x2 = F::sub(F::mul(x20, cphi), F::mul(y20, sphi));
    const T y2 = F::add(F::mul(x20, sphi), F::mul(y20, cphi));
    const T x21 = F::sub(x2, x1), y21 = F::sub(y2, y1);
    // edges of the bin (the reference recomputes them in every slab)
    T e[2][2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        T ex, ey;
        dd_det(p, dd_edge(ia + s, p.da, p.ai, p.na), ex, ey);
        e[s][0] = F::sub(F::sub(F::mul(ex, cphi), F::mul(ey, sphi)), x1);
        e[s][1] = F::sub(F::add(F::mul(ex, sphi), F::mul(ey, cphi)), y1);
    }
    const bool xdrive = dd_abs(x21) > dd_abs(y21);     // uniform: x21, y21 do not depend on the row
    const int nu = xdrive ? p.nx : p.ny, nvt = xdrive ? p.ny : p.nx;
    const T u1 = xdrive ? x1 : y1, v1 = xdrive ? y1 : x1, u21 = xdrive ? x21 : y21;
    const T ul = xdrive ? e[0][0] : e[0][1], vl = xdrive ? e[0][1] : e[0][0];
    const T ur = xdrive ? e[1][0] : e[1][1], vr = xdrive ? e[1][1] : e[1][0];
    // the reference divides inside the slab loop; the quotients do not depend on the slab
    const T r0 = F::div(vl, ul), r1 = F::div(vl, ur), r2 = F::div(vr, ul), r3 = F::div(vr, ur);
    const T hdb = F::div(p.db, (T)2);
    // the row's own part: its z slopes and length
    T rzl[R], rzr[R], len_au[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int ib = (blockIdx.y * R + r) * 32 + lane;
        const T z20 = dd_center(has[r] ? ib : 0, p.db, p.bi, p.nb);
        const T z2 = F::add(z20, off);
        const T z21 = F::sub(z2, z1);
        const T len = F::sqrt(F::add(F::add(F::mul(x21, x21), F::mul(y21, y21)), F::mul(z21, z21)));
        rzl[r] = F::div(F::sub(z21, hdb), u21);
        rzr[r] = F::div(F::add(z21, hdb), u21);
        len_au[r] = F::div(len, dd_abs(u21));
    }
    const T vhalf = (T)(nvt / 2), zhalf = (T)(p.nz / 2), uhalf = F::div((T)nu, (T)2);
    const T sad2 = F::mul(p.sad, p.sad);
    const T xhalf = (T)(p.nx / 2), yhalf = (T)(p.ny / 2);
    T acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = (T)0;
    for (int iu = 0; iu < nu; ++iu) {
        const T uc = F::sub(F::sub(F::add((T)iu, (T)0.5), uhalf), u1);
        const T c0 = F::add(F::add(F::mul(r0, uc), v1), vhalf);
        const T c1 = F::add(F::add(F::mul(r1, uc), v1), vhalf);
        const T c2 = F::add(F::add(F::mul(r2, uc), v1), vhalf);
        const T c3 = F::add(F::add(F::mul(r3, uc), v1), vhalf);
        const T vi1 = dd_min(dd_min(c0, c1), dd_min(c2, c3));
        const T vi2 = dd_max(dd_max(c0, c1), dd_max(c2, c3));
        const int va = max(0, dd_floor(vi1)), vb = min(nvt - 1, dd_floor(vi2));
        if (va > vb) continue;                      // uniform: footprint outside the grid
        T zi1[R], zi2[R], izspan[R];
        int za[R], zb[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const T czl = F::add(F::add(F::mul(rzl[r], uc), z1), zhalf);
            const T czr = F::add(F::add(F::mul(rzr[r], uc), z1), zhalf);
            zi1[r] = dd_min(czl, czr);
            zi2[r] = dd_max(czl, czr);
            za[r] = max(0, dd_floor(zi1[r]));
            zb[r] = live[r] ? min(p.nz - 1, dd_floor(zi2[r])) : -1;
            // the reference's divisions by vspan, zspan and den become
            // multiplications by reciprocals (approximate in float: <= 1 ulp each)
            izspan[r] = dd_rcp(F::sub(zi2[r], zi1[r]));
        }
        const T ivspan = dd_rcp(F::sub(vi2, vi1));
        for (int iv2 = va; iv2 <= vb; ++iv2) {
            const T wv = F::mul(F::sub(dd_min((T)iv2 + (T)1, vi2), dd_max((T)iv2, vi1)), ivspan);
            const int ix = xdrive ? iu : iv2, iy = xdrive ? iv2 : iu;
            T fw = (T)1;
            if (p.fdk) {
                // (ix + 0.5 - nx / 2): exact
                const T xc = F::sub(F::add((T)ix, (T)0.5), xhalf);
                const T yc = F::sub(F::add((T)iy, (T)0.5), yhalf);
                const T den = F::add(F::add(p.sad, F::mul(xc, cphi)), F::mul(yc, sphi));
                const T iden = dd_rcp(den);
                fw = F::mul(F::mul(sad2, iden), iden);
            }
            // the float path walks the z-fastest copy: unit z stride
            const size_t col = (size_t)iy * p.sy + (size_t)ix * p.sx;
            const size_t zs = kF32 ? 1 : (size_t)p.sz;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (FWD) {
                    // wv * (len / |u21|) * fw per voxel of the column, times wz
                    const T cw = F::mul(F::mul(wv, len_au[r]), fw);
                    const T *c = p.src + col;
                    for (int iz = za[r]; iz <= zb[r]; ++iz) {
                        const T wz = F::mul(F::sub(dd_min((T)iz + (T)1, zi2[r]), dd_max((T)iz, zi1[r])), izspan[r]);
                        acc[r] = F::add(acc[r], F::mul(__ldg(c + (size_t)iz * zs), F::mul(cw, wz)));
                    }
                } else {
                    // value * wv * (len / |u21|) * fw per voxel of the column, times wz
                    const T cw = F::mul(F::mul(F::mul(value[r], wv), len_au[r]), fw);
                    T *c = p.dst + col;
                    for (int iz = za[r]; iz <= zb[r]; ++iz) {
                        const T wz = F::mul(F::sub(dd_min((T)iz + (T)1, zi2[r]), dd_max((T)iz, zi1[r])), izspan[r]);
                        atomicAdd(c + (size_t)iz * zs, F::mul(cw, wz));
                    }
                }
            }
        }
    }
    if (FWD) {
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (has[r]) p.dst[bin[r]] = acc[r];
    }
}

static nefct_status check_dd(const nefct_dd_geom *g)
{
    if (!g) return fail(NEFCT_ERR_INVALID, "geometry is NULL");
    if (g->nx < 1 || g->ny < 1 || g->nz < 1) return fail(NEFCT_ERR_INVALID, "grid must be >= 1 voxel per axis");
    if (g->nx > (1 << 20) || g->ny > 65535 || g->nz > (1 << 20) || (long long)g->nx * g->ny * g->nz >= (1ll << 31))
        return fail(NEFCT_ERR_INVALID, "grid too large (%d x %d x %d)", g->nx, g->ny, g->nz);
    if (g->nv < 1 || !g->angles) return fail(NEFCT_ERR_INVALID, "need nv >= 1 view angles");
    if (g->na < 1 || g->nb < 1 || g->nb > 65535 * 32)
        return fail(NEFCT_ERR_INVALID, "detector must be >= 1 x 1 (got %d x %d)", g->na, g->nb);
    if (g->det_kind != NEFCT_DET_FLAT && g->det_kind != NEFCT_DET_CYL)
        return fail(NEFCT_ERR_INVALID, "det_kind must be NEFCT_DET_FLAT or NEFCT_DET_CYL");
    const float v[7] = {g->src_iso, g->src_det, g->da, g->a_offset, g->db, g->b_offset, 0.f};
    for (int i = 0; i < 6; ++i)
        if (!std::isfinite(v[i])) return fail(NEFCT_ERR_INVALID, "geometry must be finite");
    for (int i = 0; i < g->nv; ++i)
        if (!std::isfinite(g->angles[i]) || (g->z_offsets && !std::isfinite(g->z_offsets[i])))
            return fail(NEFCT_ERR_INVALID, "view %d: angle / offset not finite", i);
    return NEFCT_OK;
}

template <typename T>
static nefct_status dd_impl(const nefct_dd_geom *g, const T *src, T *dst, uint32_t flags, void *ws, size_t ws_bytes,
                            cudaStream_t s, bool forward)
{
    nefct_status st = check_dd(g);
    if (st) return st;
    if (!src || !dst) return fail(NEFCT_ERR_INVALID, "input and output must be non-NULL");
    if (flags & ~NEFCT_FDK_NO_WEIGHT) return fail(NEFCT_ERR_INVALID, "unknown flag bits 0x%x", flags);
    const bool f32 = sizeof(T) == sizeof(float);
    const size_t nvox = (size_t)g->nx * g->ny * g->nz;
    const nefct_grid gr{g->nx, g->ny, g->nz, 0.f, 0.f, 0.f, (float)g->nx, (float)g->ny, (float)g->nz};
    DDParams<T> *p = new DDParams<T>();
    p->nx = g->nx; p->ny = g->ny; p->nz = g->nz; p->na = g->na; p->nb = g->nb;
    p->cyl = g->det_kind == NEFCT_DET_CYL;
    p->fdk = !(flags & NEFCT_FDK_NO_WEIGHT);
    p->sid = g->src_det; p->sad = g->src_iso;
    p->da = g->da; p->ai = g->a_offset; p->db = g->db; p->bi = g->b_offset;
    if (f32) {
        // float: a z-fastest volume copy [y][x][z] (forward source / backward
        // accumulator), so the 32 rows of a warp touch neighbouring z
        const size_t need = nefct_dd_workspace_bytes(g);
        if (!ws || ws_bytes < need) {
            delete p;
            return fail(NEFCT_ERR_WORKSPACE, "needs %zu workspace bytes, got %zu", need, ws_bytes);
        }
        p->sx = (unsigned long long)g->nz;
        p->sy = (unsigned long long)g->nx * g->nz;
        p->sz = 1;
        if (forward) {
            st = zmajor_copy((const float *)src, (float *)ws, gr, s);
            if (st) { delete p; return st; }
            p->src = (const T *)ws;
            p->dst = dst;
        } else {
            const cudaError_t e = cudaMemsetAsync(ws, 0, need, s);
            if (e != cudaSuccess) { delete p; return cuda_fail(e, "cudaMemsetAsync"); }
            p->src = src;
            p->dst = (T *)ws;
        }
    } else {
        // double (checks and tests): the x-fastest volume in place, no workspace
        p->sx = 1;
        p->sy = (unsigned long long)g->nx;
        p->sz = (unsigned long long)g->nx * g->ny;
        p->src = src;
        p->dst = dst;
        if (!forward) {
            const cudaError_t e = cudaMemsetAsync(dst, 0, nvox * sizeof(T), s);
            if (e != cudaSuccess) { delete p; return cuda_fail(e, "cudaMemsetAsync"); }
        }
    }
    const int cols = 4;
    const int kMax = ViewTable<T>::kMax;
    for (int v0 = 0; v0 < g->nv; v0 += kMax) {
        const int nvc = std::min(kMax, g->nv - v0);
        p->v0 = v0;
        p->nvc = nvc;
        for (int i = 0; i < nvc; ++i) {
            const double a = (double)g->angles[v0 + i];
            p->tab.cs[i] = (T)cos(a);
            p->tab.sn[i] = (T)sin(a);
            p->tab.off[i] = g->z_offsets ? (T)g->z_offsets[v0 + i] : (T)0;
        }
        dim3 grid((g->na + cols - 1) / cols, (g->nb + 32 * kDDRows - 1) / (32 * kDDRows), nvc);
        if (forward) dd_kernel<T, true, kDDRows><<<grid, dim3(32, cols), 0, s>>>(*p);
        else dd_kernel<T, false, kDDRows><<<grid, dim3(32, cols), 0, s>>>(*p);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { delete p; return cuda_fail(e, forward ? "dd_kernel<forward>" : "dd_kernel<backward>"); }
    }
    delete p;
    if (f32 && !forward) return zfold((const float *)ws, (float *)dst, gr, s);
    return NEFCT_OK;
}

}  // namespace nefct

using namespace nefct;

extern "C" {

size_t nefct_dd_workspace_bytes(const nefct_dd_geom *g)
{
    if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1) return 0;
    return (size_t)g->nx * g->ny * g->nz * sizeof(float);
}

nefct_status nefct_dd_backproject(const nefct_dd_geom *g, const float *proj, float *vol, void *ws, size_t ws_bytes,
                                  void *stream)
{
    return dd_impl<float>(g, proj, vol, 0, ws, ws_bytes, (cudaStream_t)stream, false);
}

nefct_status nefct_dd_forward(const nefct_dd_geom *g, const float *vol, float *proj, uint32_t flags, void *ws,
                              size_t ws_bytes, void *stream)
{
    return dd_impl<float>(g, vol, proj, flags, ws, ws_bytes, (cudaStream_t)stream, true);
}

nefct_status nefct_dd_backward(const nefct_dd_geom *g, const float *proj, float *vol, uint32_t flags, void *ws,
                               size_t ws_bytes, void *stream)
{
    return dd_impl<float>(g, proj, vol, flags, ws, ws_bytes, (cudaStream_t)stream, false);
}

nefct_status nefct_dd_forward_f64(const nefct_dd_geom *g, const double *vol, double *proj, uint32_t flags,
                                  void *stream)
{
    return dd_impl<double>(g, vol, proj, flags, nullptr, 0, (cudaStream_t)stream, true);
}

nefct_status nefct_dd_backward_f64(const nefct_dd_geom *g, const double *proj, double *vol, uint32_t flags,
                                   void *stream)
{
    return dd_impl<double>(g, proj, vol, flags, nullptr, 0, (cudaStream_t)stream, false);
}

}  // extern "C"
