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

struct DDParams {
    int nx, ny, nz, na, nb, nvc, v0, cyl;
    float sid, sad;               // source-detector, source-axis (the reference's SID, SAD)
    float da, ai, db, bi;
    const float *proj;            // [nv][nb][na], full
    float *acc;                   // z-fastest [y][x][z]
    ViewTable<float> tab;
};

// (i + 0.5) * d + o - n * d / 2 with the reference's promotions: the first
// part in double, n * d / 2 in float (:45-60)
__device__ __forceinline__ float dd_center(int i, float d, float o, int n)
{
    const float half = __fdiv_rn(__fmul_rn((float)n, d), 2.f);
    return (float)__dsub_rn(__dadd_rn(__dmul_rn((double)i + 0.5, (double)d), (double)o), (double)half);
}

// i * d + o - n * d / 2 in float (:78-80)
__device__ __forceinline__ float dd_edge(int i, float d, float o, int n)
{
    return __fsub_rn(__fadd_rn(__fmul_rn((float)i, d), o), __fdiv_rn(__fmul_rn((float)n, d), 2.f));
}

// cos/sin of a detector angle: the double-precision functions, rounded
__device__ __forceinline__ void dd_trig(float a, float &c, float &s)
{
    double sd, cd;
    sincos((double)a, &sd, &cd);
    c = (float)cd;
    s = (float)sd;
}

// detector point (x20, y20) of lateral coordinate a (flat: a is the offset
// along the detector; cylindrical: the angle)
__device__ __forceinline__ void dd_det(const DDParams &p, float a, float &x20, float &y20)
{
    if (p.cyl) {
        float c, s;
        dd_trig(a, c, s);
        x20 = __fsub_rn(__fmul_rn(p.sid, c), p.sad);
        y20 = __fmul_rn(p.sid, s);
    } else {
        x20 = __fsub_rn(p.sid, p.sad);
        y20 = a;
    }
}

__device__ __forceinline__ float dd_min(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float dd_max(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float dd_abs(float a) { return a > 0.f ? a : -a; }

__global__ void __launch_bounds__(256) dd_backproject_kernel(const __grid_constant__ DDParams p)
{
    const int lane = threadIdx.x;
    const int ia = blockIdx.x * blockDim.y + threadIdx.y;
    const int ib = blockIdx.y * 32 + lane;
    const int iv = blockIdx.z;
    if (ia >= p.na) return;                       // uniform across the warp
    const bool has = ib < p.nb;
    const float value = has ? p.proj[((size_t)(p.v0 + iv) * p.nb + ib) * p.na + ia] : 0.f;
    if (!__any_sync(0xffffffffu, value != 0.f)) return;
    const bool live = value != 0.f;

    const float cphi = p.tab.cs[iv], sphi = p.tab.sn[iv], off = p.tab.off[iv];
    const float x1 = __fmul_rn(-p.sad, cphi), y1 = __fmul_rn(-p.sad, sphi), z1 = off;
    float x20, y20;
    dd_det(p, dd_center(ia, p.da, p.ai, p.na), x20, y20);
    const float z20 = dd_center(has ? ib : 0, p.db, p.bi, p.nb);
    const float x2 = __fsub_rn(__fmul_rn(x20, cphi), __fmul_rn(y20, sphi));
    const float y2 = __fadd_rn(__fmul_rn(x20, sphi), __fmul_rn(y20, cphi));
    const float z2 = __fadd_rn(z20, off);
    const float x21 = __fsub_rn(x2, x1), y21 = __fsub_rn(y2, y1), z21 = __fsub_rn(z2, z1);
    // edges of the bin (the reference recomputes them in every slab)
    float e[2][2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        float ex, ey;
        dd_det(p, dd_edge(ia + s, p.da, p.ai, p.na), ex, ey);
        e[s][0] = __fsub_rn(__fsub_rn(__fmul_rn(ex, cphi), __fmul_rn(ey, sphi)), x1);
        e[s][1] = __fsub_rn(__fadd_rn(__fmul_rn(ex, sphi), __fmul_rn(ey, cphi)), y1);
    }
    const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x21, x21), __fmul_rn(y21, y21)), __fmul_rn(z21, z21)));
    const bool xdrive = dd_abs(x21) > dd_abs(y21);     // uniform: x21, y21 do not depend on the row
    const int nu = xdrive ? p.nx : p.ny, nvt = xdrive ? p.ny : p.nx;
    const float u1 = xdrive ? x1 : y1, v1 = xdrive ? y1 : x1, u21 = xdrive ? x21 : y21;
    const float ul = xdrive ? e[0][0] : e[0][1], vl = xdrive ? e[0][1] : e[0][0];
    const float ur = xdrive ? e[1][0] : e[1][1], vr = xdrive ? e[1][1] : e[1][0];
    // the reference divides inside the slab loop; the quotients do not depend on the slab
    const float r0 = __fdiv_rn(vl, ul), r1 = __fdiv_rn(vl, ur), r2 = __fdiv_rn(vr, ul), r3 = __fdiv_rn(vr, ur);
    const float hdb = __fdiv_rn(p.db, 2.f);
    const float rzl = __fdiv_rn(__fsub_rn(z21, hdb), u21), rzr = __fdiv_rn(__fadd_rn(z21, hdb), u21);
    const float vhalf = (float)(nvt / 2), zhalf = (float)(p.nz / 2), uhalf = __fdiv_rn((float)nu, 2.f);
    const float len_au = __fdiv_rn(len, dd_abs(u21));
    const float sad2 = __fmul_rn(p.sad, p.sad);
    const float xhalf = (float)(p.nx / 2), yhalf = (float)(p.ny / 2);
    const unsigned zs = (unsigned)p.nz;
    for (int iu = 0; iu < nu; ++iu) {
        const float uc = __fsub_rn(__fsub_rn(__fadd_rn((float)iu, 0.5f), uhalf), u1);
        const float c0 = __fadd_rn(__fadd_rn(__fmul_rn(r0, uc), v1), vhalf);
        const float c1 = __fadd_rn(__fadd_rn(__fmul_rn(r1, uc), v1), vhalf);
        const float c2 = __fadd_rn(__fadd_rn(__fmul_rn(r2, uc), v1), vhalf);
        const float c3 = __fadd_rn(__fadd_rn(__fmul_rn(r3, uc), v1), vhalf);
        const float vi1 = dd_min(dd_min(c0, c1), dd_min(c2, c3));
        const float vi2 = dd_max(dd_max(c0, c1), dd_max(c2, c3));
        const int va = max(0, (int)floorf(vi1)), vb = min(nvt - 1, (int)floorf(vi2));
        if (va > vb) continue;                      // uniform: footprint outside the grid
        const float czl = __fadd_rn(__fadd_rn(__fmul_rn(rzl, uc), z1), zhalf);
        const float czr = __fadd_rn(__fadd_rn(__fmul_rn(rzr, uc), z1), zhalf);
        const float zi1 = dd_min(czl, czr), zi2 = dd_max(czl, czr);
        const int za = max(0, (int)floorf(zi1)), zb = live ? min(p.nz - 1, (int)floorf(zi2)) : -1;
        const float vspan = __fsub_rn(vi2, vi1), zspan = __fsub_rn(zi2, zi1);
        // the reference's divisions by vspan, zspan and den become
        // multiplications by approximate reciprocals (<= 1 ulp each)
        const float ivspan = rcp_approx(vspan), izspan = rcp_approx(zspan);
        for (int iv2 = va; iv2 <= vb; ++iv2) {
            const float wv = __fmul_rn(__fsub_rn(dd_min((float)iv2 + 1.0f, vi2), dd_max((float)iv2, vi1)), ivspan);
            const int ix = xdrive ? iu : iv2, iy = xdrive ? iv2 : iu;
            // (ix + 0.5 - nx / 2): exact in float
            const float xc = __fsub_rn(__fadd_rn((float)ix, 0.5f), xhalf);
            const float yc = __fsub_rn(__fadd_rn((float)iy, 0.5f), yhalf);
            const float den = __fadd_rn(__fadd_rn(p.sad, __fmul_rn(xc, cphi)), __fmul_rn(yc, sphi));
            const float iden = rcp_approx(den);
            const float fw = __fmul_rn(__fmul_rn(sad2, iden), iden);
            // value * wv * (len / |u21|) * fw per voxel of the column, times wz
            const float cw = __fmul_rn(__fmul_rn(__fmul_rn(value, wv), len_au), fw);
            float *col = p.acc + ((size_t)iy * p.nx + ix) * zs;
            for (int iz = za; iz <= zb; ++iz) {
                const float wz = __fmul_rn(__fsub_rn(dd_min((float)iz + 1.0f, zi2), dd_max((float)iz, zi1)), izspan);
                atomicAdd(col + iz, __fmul_rn(cw, wz));
            }
        }
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
    nefct_status st = check_dd(g);
    if (st) return st;
    if (!proj || !vol) return fail(NEFCT_ERR_INVALID, "proj and vol must be non-NULL");
    const size_t need = nefct_dd_workspace_bytes(g);
    if (!ws || ws_bytes < need) return fail(NEFCT_ERR_WORKSPACE, "needs %zu workspace bytes, got %zu", need, ws_bytes);
    cudaStream_t s = (cudaStream_t)stream;
    NEFCT_CHECK_CUDA(cudaMemsetAsync(ws, 0, need, s));
    DDParams *p = new DDParams();
    p->nx = g->nx; p->ny = g->ny; p->nz = g->nz; p->na = g->na; p->nb = g->nb;
    p->cyl = g->det_kind == NEFCT_DET_CYL;
    p->sid = g->src_det; p->sad = g->src_iso;
    p->da = g->da; p->ai = g->a_offset; p->db = g->db; p->bi = g->b_offset;
    p->proj = proj;
    p->acc = (float *)ws;
    const int cols = 4;
    const int kMax = ViewTable<float>::kMax;
    for (int v0 = 0; v0 < g->nv; v0 += kMax) {
        const int nvc = std::min(kMax, g->nv - v0);
        p->v0 = v0;
        p->nvc = nvc;
        for (int i = 0; i < nvc; ++i) {
            const double a = (double)g->angles[v0 + i];
            p->tab.cs[i] = (float)cos(a);
            p->tab.sn[i] = (float)sin(a);
            p->tab.off[i] = g->z_offsets ? g->z_offsets[v0 + i] : 0.f;
        }
        dim3 grid((g->na + cols - 1) / cols, (g->nb + 31) / 32, nvc);
        dd_backproject_kernel<<<grid, dim3(32, cols), 0, s>>>(*p);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { delete p; return cuda_fail(e, "dd_backproject_kernel"); }
    }
    delete p;
    const nefct_grid gr{g->nx, g->ny, g->nz, 0.f, 0.f, 0.f, (float)g->nx, (float)g->ny, (float)g->nz};
    return zfold((const float *)ws, vol, gr, s);
}

}  // extern "C"
