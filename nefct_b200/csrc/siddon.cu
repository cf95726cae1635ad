// Cone-beam and LOR Siddon projectors on sm_100a: host side of the cone-beam
// projector (validation, per-view tables, workspace, transposes, the
// deterministic transpose), the intersection count, the LOR pair and the
// C-ABI entry points (declared in include/nefct_b200.h).  The cone-beam
// kernels themselves are in cb_kernels.cuh.
//
// Neighbouring rays of a warp cross a driving slab at neighbouring
// transverse positions; with the transverse axis contiguous in memory a
// warp's gather touches one or two 128-byte lines.  That holds for y-driven
// rays in the x-fastest volume; x-driven rays read a y-fastest copy of the
// volume (one transpose per call, in the caller's workspace).
#include <math.h>
#include <algorithm>
#include <mutex>
#include <type_traits>

#include "cb_kernels.cuh"

namespace nefct {

template <bool DIV>
__global__ void __launch_bounds__(256) cb_count_kernel(const __grid_constant__ CBParams<float> p)
{
    int ia, ib, iv;
    cb_cell(p, ia, ib, iv);
    unsigned n = 0;
    if (ia < p.na && ib < p.nb) {
        float r[6];
        cb_ray(p, ia, ib, iv, r);
        Walk<float> w;
        if (setup_walk(p.g, r, p.flags, w)) n = count_walk<float, DIV>(w, p.g);
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(p.count, (unsigned long long)n);
}

// ---------------- deterministic transpose (fixed point) ----------------

template <bool DIV>
__global__ void __launch_bounds__(256) cb_backward_fixed_kernel(const __grid_constant__ CBParams<float> p)
{
    int ia, ib, iv;
    cb_cell(p, ia, ib, iv);
    if (ia >= p.na || ib >= p.nb) return;
    const float y = cb_sino_value(p, ia, ib, iv);
    if (y == 0.f) return;
    float r[6];
    cb_ray(p, ia, ib, iv, r);
    Walk<float> w;
    if (!setup_walk(p.g, r, p.flags, w)) return;
    const float scale = *p.fix_scale;
    const int sw = p.g.nx * p.g.ny;
    if (!w.xdrive) scatter_walk_fixed<float, DIV, true>(w, p.g, p.fix, p.g.nx, 1, sw, y, scale);
    else if (p.fixT) scatter_walk_fixed<float, DIV, true>(w, p.g, p.fixT, p.g.ny, 1, sw, y, scale);
    else scatter_walk_fixed<float, DIV, false>(w, p.g, p.fix, 1, p.g.nx, sw, y, scale);
}

// Column-warp variant: 64-bit fixed-point reductions into a z-fastest
// accumulator (the same per-contribution integers as the thread walk, so the
// integer sums and the result are bitwise the same).
template <bool DIV>
__global__ void __launch_bounds__(256) cb_colwarp_fixed_kernel(const __grid_constant__ CBParams<float> p)
{
    const int lane = threadIdx.x;
    const int ia = blockIdx.x * blockDim.y + threadIdx.y;
    int ib, iv;
    if (p.band_major) { iv = blockIdx.y; ib = blockIdx.z * 32 + lane; }
    else { ib = blockIdx.y * 32 + lane; iv = blockIdx.z; }
    if (ia >= p.na) return;                       // uniform across the warp
    const bool has = ib < p.nb;
    const float y = has ? cb_sino_value(p, ia, ib, iv) : 0.f;
    float r[6];
    cb_ray(p, ia, has ? ib : 0, iv, r);
    colwarp_lane<DIV, false, true>(p.g, r, has, p.flags, nullptr, nullptr, y, nullptr, p.fix, *p.fix_scale);
}

// vol[z][y][x] = accZ[y][x][z] / scale (the integer sums of the column warps)
__global__ void __launch_bounds__(256) fixed_zfold_kernel(const unsigned long long *__restrict__ acc, int nx, int ny,
                                                          int nz, const float *scale, float *__restrict__ vol)
{
    __shared__ unsigned long long tile[32][33];
    const int y = blockIdx.z, x0 = blockIdx.x * 32, z0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + j, z = z0 + threadIdx.x;
        if (x < nx && z < nz) tile[j][threadIdx.x] = acc[((size_t)y * nx + x) * nz + z];
    }
    __syncthreads();
    const double inv = 1.0 / (double)*scale;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + threadIdx.x, z = z0 + j;
        if (x < nx && z < nz) vol[((size_t)z * ny + y) * nx + x] = (float)((double)(long long)tile[threadIdx.x][j] * inv);
    }
}

// max |x| as float bits (non-negative floats order like their bit patterns)
__global__ void __launch_bounds__(256) maxabs_kernel(const float *__restrict__ x, size_t n, unsigned *out)
{
    unsigned m = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = max(m, __float_as_uint(fabsf(x[i])));
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// scale = 2^k with k the largest integer such that bound * max|y| * 2^k <= 2^61,
// where bound >= (rays) * (largest weight); then no per-voxel sum of
// |contribution| * scale can exceed 2^61.
__global__ void fixed_scale_kernel(const unsigned *maxbits, double bound, float *scale)
{
    const double B = bound * (double)__uint_as_float(*maxbits);
    int k = 0;
    if (B > 0.0 && B < 1e300) k = (int)floor(61.0 - log2(B));
    k = max(-126, min(127, k));
    *scale = ldexpf(1.0f, k);
}

// vol[z][y][x] = (accN[z][y][x] + accT[z][x][y]) / scale, integer sum first
__global__ void __launch_bounds__(256) fixed_fold_kernel(const unsigned long long *__restrict__ accN,
                                                         const unsigned long long *__restrict__ accT, int nx, int ny,
                                                         const float *scale, float *__restrict__ vol)
{
    __shared__ unsigned long long tile[32][33];
    const size_t plane = (size_t)nx * ny * blockIdx.z;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    if (accT) {
        for (int j = threadIdx.y; j < 32; j += 8) {
            const int y = y0 + threadIdx.x, x = x0 + j;
            if (x < nx && y < ny) tile[j][threadIdx.x] = accT[plane + (size_t)x * ny + y];
        }
    }
    __syncthreads();
    const double inv = 1.0 / (double)*scale;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + threadIdx.x, y = y0 + j;
        if (x < nx && y < ny) {
            unsigned long long v = accN[plane + (size_t)y * nx + x];
            if (accT) v += tile[threadIdx.x][j];
            vol[plane + (size_t)y * nx + x] = (float)((double)(long long)v * inv);
        }
    }
}

// ---------------- LOR projector pair (cpp/siddon) ----------------

template <typename T> struct LorParams {
    GridDev<T> g;
    const T *lors;
    long long n;
    uint32_t flags;
    const T *vol;
    const T *vals;
    T *out;
    const int32_t *order;     // walk order (a permutation of 0..n-1), or nullptr
};

// The walk visits lines in `order` so that a warp's 32 lines are nearly
// parallel neighbours (similar trip counts, nearby voxels); results stay at
// each line's own index.
template <typename T, bool DIV, bool Q5>
__global__ void __launch_bounds__(256) lor_forward_kernel(const __grid_constant__ LorParams<T> p)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < p.n;
         t += (long long)gridDim.x * blockDim.x) {
        const long long i = p.order ? (long long)p.order[t] : t;
        T r[6];
        for (int j = 0; j < 6; ++j) r[j] = p.lors[j * p.n + i];
        Walk<T> w;
        T acc = (T)0;
        if (setup_walk(p.g, r, p.flags, w)) {
            const int sw = p.g.nx * p.g.ny;
            acc = w.xdrive ? gather_walk<T, DIV, false, Q5>(w, p.g, p.vol, 1, p.g.nx, sw)
                           : gather_walk<T, DIV, true, Q5>(w, p.g, p.vol, p.g.nx, 1, sw);
        }
        p.out[i] = acc;
    }
}

template <typename T, bool DIV, bool Q5>
__global__ void __launch_bounds__(256) lor_backward_kernel(const __grid_constant__ LorParams<T> p)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < p.n;
         t += (long long)gridDim.x * blockDim.x) {
        const long long i = p.order ? (long long)p.order[t] : t;
        const T y = p.vals[i];
        if (y == (T)0) continue;
        T r[6];
        for (int j = 0; j < 6; ++j) r[j] = p.lors[j * p.n + i];
        Walk<T> w;
        if (!setup_walk(p.g, r, p.flags, w)) continue;
        const int sw = p.g.nx * p.g.ny;
        if (w.xdrive) scatter_walk<T, DIV, false, Q5>(w, p.g, p.out, 1, p.g.nx, sw, y);
        else scatter_walk<T, DIV, true, Q5>(w, p.g, p.out, p.g.nx, 1, sw, y);
    }
}

// Ordering key of a line (31 bits, larger = later): driving axis, in-plane
// direction folded to [0, pi), signed distance of the in-plane line from the
// grid centre, z where the line passes the centre, and z slope.  Lines with
// equal keys are nearly parallel neighbours.
__global__ void __launch_bounds__(256) lor_key_kernel(const __grid_constant__ LorParams<float> p, int32_t *keys)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < p.n;
         i += (long long)gridDim.x * blockDim.x) {
        const float x1 = p.lors[i] - p.g.cx, y1 = p.lors[p.n + i] - p.g.cy, z1 = p.lors[2 * p.n + i] - p.g.cz;
        const float dx = p.lors[3 * p.n + i] - p.g.cx - x1, dy = p.lors[4 * p.n + i] - p.g.cy - y1;
        const float dz = p.lors[5 * p.n + i] - p.g.cz - z1;
        const float sx = (float)p.g.nx * p.g.dx_, sy = p.g.dy * (float)p.g.ny * p.g.dx_;
        const float sz = p.g.dz * (float)p.g.nz * p.g.dx_;
        const float lxy = sqrtf(dx * dx + dy * dy);
        const unsigned xdrive = fabsf(dx) >= fabsf(dy);
        float th = atan2f(dy, dx);
        if (th < 0.f) th += 3.14159265f;
        if (th >= 3.14159265f) th -= 3.14159265f;
        const float ux = lxy > 0.f ? dx / lxy : 1.f, uy = lxy > 0.f ? dy / lxy : 0.f;
        const float rad = 0.5f * sqrtf(sx * sx + sy * sy) + 1e-6f;
        const float perp = (x1 * uy - y1 * ux) / rad;                 // [-1, 1] for lines through the grid
        const float along = -(x1 * ux + y1 * uy);                     // parameter (in-plane length) of the centre
        const float slope = lxy > 0.f ? dz / lxy : 0.f;
        const float zc = (z1 + slope * along) / (sz + 1e-6f);         // about [-0.5, 0.5] inside
        auto q = [](float v, float lo, float hi, int bits) {
            const float f = fminf(fmaxf((v - lo) / (hi - lo), 0.f), 1.f);
            return (unsigned)fminf(f * (float)(1 << bits), (float)((1 << bits) - 1));
        };
        // z centre and slope interleaved bit by bit (a Z-order curve): the
        // lines of one direction and offset bin fall into warps of similar
        // z entry and exit, so the walks of a warp have similar lengths
        const unsigned zq = q(zc, -1.f, 1.f, 7), sq = q(atanf(slope), -1.5708f, 1.5708f, 7);
        unsigned zs = 0;
#pragma unroll
        for (int b = 0; b < 7; ++b) zs |= ((zq >> b) & 1u) << (2 * b + 1) | ((sq >> b) & 1u) << (2 * b);
        const unsigned k = (xdrive << 30) | (q(th, 0.f, 3.14159265f, 8) << 22) | (q(perp, -1.f, 1.f, 8) << 14) | zs;
        keys[i] = (int32_t)k;
    }
}

// ---------------- host side ----------------

static const uint32_t kWalkFlags = NEFCT_TIE_GT | NEFCT_SKIP_SHORT | NEFCT_NO_INV_L2 | NEFCT_Q5 |
                                   NEFCT_Q8_INDEX | NEFCT_NO_TRANSPOSE | NEFCT_DETERMINISTIC | NEFCT_EXACT;

// Flags of the cone-beam calls: the walk switches except NEFCT_Q5, a quirk of
// the LOR projector (cpp/siddon) that no cone-beam walk applies.
static nefct_status check_cb_flags(uint32_t flags)
{
    if (flags & ~kWalkFlags) return fail(NEFCT_ERR_INVALID, "unknown flag bits 0x%x", flags & ~kWalkFlags);
    if (flags & NEFCT_Q5)
        return fail(NEFCT_ERR_UNSUPPORTED, "NEFCT_Q5 belongs to the LOR projector; the cone-beam walks do not take it");
    return NEFCT_OK;
}

static nefct_status check_grid(const nefct_grid &g)
{
    if (g.nx < 1 || g.ny < 1 || g.nz < 1)
        return fail(NEFCT_ERR_INVALID, "grid dimensions must be >= 1 (got %d x %d x %d)", g.nx, g.ny, g.nz);
    if (g.nx > (1 << 20) || g.ny > (1 << 20) || g.nz > (1 << 20))
        return fail(NEFCT_ERR_INVALID, "grid dimensions must be <= 2^20 (got %d x %d x %d)", g.nx, g.ny, g.nz);
    if ((long long)g.nx * g.ny * g.nz >= (1ll << 31))
        return fail(NEFCT_ERR_INVALID, "grid has %lld voxels; at most 2^31-1 are supported",
                    (long long)g.nx * g.ny * g.nz);
    const float v[6] = {g.cx, g.cy, g.cz, g.sx, g.sy, g.sz};
    for (int i = 0; i < 6; ++i)
        if (!std::isfinite(v[i])) return fail(NEFCT_ERR_INVALID, "grid centre/size must be finite");
    if (!(g.sx > 0.f && g.sy > 0.f && g.sz > 0.f)) return fail(NEFCT_ERR_INVALID, "grid size must be > 0");
    return NEFCT_OK;
}

nefct_status check_cb_geom(const nefct_cb_geom *g)
{
    if (!g) return fail(NEFCT_ERR_INVALID, "geometry is NULL");
    nefct_status st = check_grid(g->grid);
    if (st) return st;
    if (g->nv < 1 || !g->angles) return fail(NEFCT_ERR_INVALID, "need nv >= 1 view angles (nv=%d)", g->nv);
    if (g->na < 1 || g->nb < 1) return fail(NEFCT_ERR_INVALID, "detector must be >= 1 x 1 (got %d x %d)", g->na, g->nb);
    if ((long long)g->na * g->nb * g->nv >= (1ll << 40))
        return fail(NEFCT_ERR_INVALID, "sinogram too large");
    if ((long long)g->na * g->nb >= (1ll << 31)) return fail(NEFCT_ERR_INVALID, "detector too large");
    if (g->nb > 65535 || g->grid.nz > 65535)
        return fail(NEFCT_ERR_INVALID, "detector rows and nz must be <= 65535 (got %d, %d)", g->nb, g->grid.nz);
    if (g->det_kind != NEFCT_DET_FLAT && g->det_kind != NEFCT_DET_CYL)
        return fail(NEFCT_ERR_INVALID, "det_kind must be NEFCT_DET_FLAT or NEFCT_DET_CYL (got %d)", g->det_kind);
    const float v[6] = {g->src_iso, g->src_det, g->da, g->a_shift, g->db, g->b_shift};
    for (int i = 0; i < 6; ++i)
        if (!std::isfinite(v[i])) return fail(NEFCT_ERR_INVALID, "scanner geometry must be finite");
    if (g->da == 0.f || g->db == 0.f) return fail(NEFCT_ERR_INVALID, "detector pitch must be non-zero");
    for (int i = 0; i < g->nv; ++i) {
        if (!std::isfinite(g->angles[i])) return fail(NEFCT_ERR_INVALID, "angle %d is not finite", i);
        if (g->z_offsets && !std::isfinite(g->z_offsets[i]))
            return fail(NEFCT_ERR_INVALID, "z offset %d is not finite", i);
    }
    return NEFCT_OK;
}

template <typename T> static void fill_cb_params(CBParams<T> &p, const nefct_cb_geom *g, uint32_t flags)
{
    p.g = make_grid_dev<T>(g->grid);
    p.na = g->na; p.nb = g->nb; p.nv_total = g->nv;
    p.rg = make_ray_geom<T>(*g);
    p.flags = flags;
}

// cos/sin of the view angles from the double-precision functions, rounded.
template <typename T> static void fill_views(CBParams<T> &p, const nefct_cb_geom *g, int v0, int nvc)
{
    p.v0 = v0; p.nvc = nvc;
    for (int i = 0; i < nvc; ++i) {
        const double a = (double)g->angles[v0 + i];
        p.tab.cs[i] = (T)cos(a);
        p.tab.sn[i] = (T)sin(a);
        p.tab.off[i] = g->z_offsets ? (T)g->z_offsets[v0 + i] : (T)0;
    }
}

// volZ[y][x][z] = vol[z][y][x]  (32x32 tiles of each y plane)
__global__ void __launch_bounds__(256) zmajor_kernel(const float *__restrict__ in, float *__restrict__ out, int nx,
                                                     int ny, int nz)
{
    __shared__ float tile[32][33];
    const int y = blockIdx.z, x0 = blockIdx.x * 32, z0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + threadIdx.x, z = z0 + j;
        if (x < nx && z < nz) tile[j][threadIdx.x] = in[((size_t)z * ny + y) * nx + x];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + j, z = z0 + threadIdx.x;
        if (x < nx && z < nz) out[((size_t)y * nx + x) * nz + z] = tile[threadIdx.x][j];
    }
}

// vol[z][y][x] = accZ[y][x][z]
__global__ void __launch_bounds__(256) zfold_kernel(const float *__restrict__ acc, float *__restrict__ vol, int nx,
                                                    int ny, int nz)
{
    __shared__ float tile[32][33];
    const int y = blockIdx.z, x0 = blockIdx.x * 32, z0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + j, z = z0 + threadIdx.x;
        if (x < nx && z < nz) tile[j][threadIdx.x] = acc[((size_t)y * nx + x) * nz + z];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + threadIdx.x, z = z0 + j;
        if (x < nx && z < nz) vol[((size_t)z * ny + y) * nx + x] = tile[threadIdx.x][j];
    }
}

// z-fastest copy [y][x][z] of an x-fastest volume (column-warp forward)
nefct_status zmajor_copy(const float *in, float *out, const nefct_grid &g, cudaStream_t s)
{
    dim3 grid((g.nx + 31) / 32, (g.nz + 31) / 32, g.ny);
    zmajor_kernel<<<grid, dim3(32, 8), 0, s>>>(in, out, g.nx, g.ny, g.nz);
    NEFCT_CHECK_LAUNCH("zmajor_kernel");
    return NEFCT_OK;
}

// vol = the x-fastest layout of the z-fastest accumulator (column-warp transpose)
nefct_status zfold(const float *acc, float *vol, const nefct_grid &g, cudaStream_t s)
{
    dim3 grid((g.nx + 31) / 32, (g.nz + 31) / 32, g.ny);
    zfold_kernel<<<grid, dim3(32, 8), 0, s>>>(acc, vol, g.nx, g.ny, g.nz);
    NEFCT_CHECK_LAUNCH("zfold_kernel");
    return NEFCT_OK;
}

template <typename T>
static nefct_status transpose_xy(const T *in, T *out, const nefct_grid &g, cudaStream_t s)
{
    dim3 grid((g.nx + 31) / 32, (g.ny + 31) / 32, g.nz);
    transpose_xy_kernel<T><<<grid, dim3(32, 8), 0, s>>>(in, out, g.nx, g.ny);
    NEFCT_CHECK_LAUNCH("transpose_xy_kernel");
    return NEFCT_OK;
}

// Launches of the forward / transpose kernels for one problem whose volume
// copy (forward) or accumulator (transpose) is given -- y-fastest for the
// thread walk, z-fastest for column warps (colwarp); no transpose, memset or
// fold.  Used by the batch's per-problem strategy.
nefct_status cb_forward_launches(const nefct_cb_geom *g, const float *vol, const float *volT, float *sino,
                                 uint32_t flags, cudaStream_t s, bool colwarp)
{
    CBParams<float> p;
    fill_cb_params(p, g, flags);
    p.vol = vol;
    p.volT = volT;
    p.out = sino;
    for (int v0 = 0; v0 < g->nv; v0 += ViewTable<float>::kMax) {
        const int nvc = std::min(ViewTable<float>::kMax, g->nv - v0);
        fill_views(p, g, v0, nvc);
        const cudaError_t e = cb_launch_forward<float>(p, g->na, g->nb, nvc, flags, s, colwarp);
        if (e != cudaSuccess) return cuda_fail(e, "cb_forward_kernel");
    }
    return NEFCT_OK;
}

nefct_status cb_backward_launches(const nefct_cb_geom *g, const float *sino, float *out, float *outT,
                                  uint32_t flags, cudaStream_t s, bool colwarp)
{
    CBParams<float> p;
    fill_cb_params(p, g, flags);
    p.sino = sino;
    p.out = out;
    p.outT = outT;
    for (int v0 = 0; v0 < g->nv; v0 += ViewTable<float>::kMax) {
        const int nvc = std::min(ViewTable<float>::kMax, g->nv - v0);
        fill_views(p, g, v0, nvc);
        const cudaError_t e = cb_launch_backward<float>(p, g->na, g->nb, nvc, flags, s, colwarp);
        if (e != cudaSuccess) return cuda_fail(e, "cb_backward_kernel");
    }
    return NEFCT_OK;
}

template <typename T>
static nefct_status cb_forward_impl(const nefct_cb_geom *g, const T *vol, T *sino, uint32_t flags, void *ws,
                                    size_t wsb, cudaStream_t s)
{
    nefct_status st = check_cb_geom(g);
    if (st) return st;
    if (!vol || !sino) return fail(NEFCT_ERR_INVALID, "vol and sino must be non-NULL");
    if ((st = check_cb_flags(flags))) return st;
    CBParams<T> *p = new CBParams<T>();
    fill_cb_params(*p, g, flags);
    p->vol = vol;
    p->out = sino;
    const size_t nvox = (size_t)g->grid.nx * g->grid.ny * g->grid.nz;
    const bool cw = cb_use_colwarp<T>(g->grid, flags, true);
    if (!(flags & NEFCT_NO_TRANSPOSE)) {
        if (!ws || wsb < nvox * sizeof(T)) {
            delete p;
            return fail(NEFCT_ERR_WORKSPACE, "forward needs %zu workspace bytes, got %zu", nvox * sizeof(T), wsb);
        }
        if constexpr (std::is_same<T, float>::value) {
            if (cw) st = zmajor_copy(vol, (float *)ws, g->grid, s);
            else st = transpose_xy(vol, (T *)ws, g->grid, s);
        } else {
            st = transpose_xy(vol, (T *)ws, g->grid, s);
        }
        if (st) { delete p; return st; }
        p->volT = (const T *)ws;
    }
    const int kMax = ViewTable<T>::kMax;
    for (int v0 = 0; v0 < g->nv; v0 += kMax) {
        const int nvc = std::min(kMax, g->nv - v0);
        fill_views(*p, g, v0, nvc);
        cudaError_t e = cb_launch_forward<T>(*p, g->na, g->nb, nvc, flags, s, cw);
        if (e != cudaSuccess) { delete p; return cuda_fail(e, "cb_forward_kernel"); }
    }
    delete p;
    return NEFCT_OK;
}

// Upper bound of (rays) x (largest contribution weight) for the fixed-point
// scale: |kv| <= 1 by the choice of driving axis; the transverse
// source-detector distance is >= src_det (flat: sqrt(src_det^2 + a^2);
// cylindrical: exactly src_det), so |kw| <= sqrt(2) max|b| / src_det and
// L >= src_det / dx in voxel units.
static double fixed_bound(const nefct_cb_geom *g, uint32_t flags)
{
    const double dx = (double)g->grid.sx / g->grid.nx;
    const double half = g->nb * (double)g->db / 2.0;
    const double b0 = fabs((0.0 + g->b_shift) * g->db - half);
    const double b1 = fabs((g->nb - 1.0 + g->b_shift) * g->db - half);
    const double kw = sqrt(2.0) * std::max(b0, b1) / g->src_det;
    double W = sqrt(2.0 + kw * kw) * dx;
    if (!(flags & NEFCT_NO_INV_L2)) W *= (dx / g->src_det) * (dx / g->src_det);
    return (double)g->na * g->nb * g->nv * W * 1.001;
}

size_t cb_fixed_workspace(const nefct_cb_geom *g, uint32_t flags)
{
    const size_t nvox = (size_t)g->grid.nx * g->grid.ny * g->grid.nz;
    return 256 + nvox * sizeof(unsigned long long) * ((flags & NEFCT_NO_TRANSPOSE) ? 1 : 2);
}

static nefct_status cb_backward_fixed_impl(const nefct_cb_geom *g, const float *sino, float *vol, uint32_t flags,
                                           void *ws, size_t wsb, cudaStream_t s)
{
    if (flags & NEFCT_EXACT)
        return fail(NEFCT_ERR_UNSUPPORTED, "NEFCT_EXACT is not available with NEFCT_DETERMINISTIC");
    if (!(g->src_det > 0.f)) return fail(NEFCT_ERR_INVALID, "deterministic transpose needs src_det > 0");
    const size_t nvox = (size_t)g->grid.nx * g->grid.ny * g->grid.nz;
    const bool tr = !(flags & NEFCT_NO_TRANSPOSE);
    const size_t need = cb_fixed_workspace(g, flags);
    if (!ws || wsb < need)
        return fail(NEFCT_ERR_WORKSPACE, "deterministic backward needs %zu workspace bytes, got %zu", need, wsb);
    unsigned char *w = (unsigned char *)ws;
    unsigned *maxbits = (unsigned *)w;
    float *scale = (float *)(w + 16);
    unsigned long long *accN = (unsigned long long *)(w + 256);
    unsigned long long *accT = tr ? accN + nvox : nullptr;
    NEFCT_CHECK_CUDA(cudaMemsetAsync(w, 0, need, s));
    const size_t ns = (size_t)g->na * g->nb * g->nv;
    maxabs_kernel<<<(unsigned)std::min<size_t>((ns + 255) / 256, 148 * 16), 256, 0, s>>>(sino, ns, maxbits);
    NEFCT_CHECK_LAUNCH("maxabs_kernel");
    fixed_scale_kernel<<<1, 1, 0, s>>>(maxbits, fixed_bound(g, flags), scale);
    NEFCT_CHECK_LAUNCH("fixed_scale_kernel");
    CBParams<float> p;
    fill_cb_params(p, g, flags);
    p.sino = sino;
    p.fix = accN;
    p.fixT = accT;
    p.fix_scale = scale;
    // column warps reduce everything into accN in z-fastest order
    const bool cw = tr && cb_use_colwarp<float>(g->grid, flags & ~NEFCT_DETERMINISTIC, false);
    for (int v0 = 0; v0 < g->nv; v0 += ViewTable<float>::kMax) {
        const int nvc = std::min(ViewTable<float>::kMax, g->nv - v0);
        fill_views(p, g, v0, nvc);
        dim3 grid, block;
        if (cw) {
            cb_colwarp_shape(p, g->na, g->nb, nvc, grid, block);
            if (cubic(p.g)) cb_colwarp_fixed_kernel<false><<<grid, block, 0, s>>>(p);
            else cb_colwarp_fixed_kernel<true><<<grid, block, 0, s>>>(p);
            NEFCT_CHECK_LAUNCH("cb_colwarp_fixed_kernel");
            continue;
        }
        cb_shape(p, g->na, g->nb, nvc, grid, block);
        if (cubic(p.g)) cb_backward_fixed_kernel<false><<<grid, block, 0, s>>>(p);
        else cb_backward_fixed_kernel<true><<<grid, block, 0, s>>>(p);
        NEFCT_CHECK_LAUNCH("cb_backward_fixed_kernel");
    }
    if (cw) {
        dim3 grid((g->grid.nx + 31) / 32, (g->grid.nz + 31) / 32, g->grid.ny);
        fixed_zfold_kernel<<<grid, dim3(32, 8), 0, s>>>(accN, g->grid.nx, g->grid.ny, g->grid.nz, scale, vol);
        NEFCT_CHECK_LAUNCH("fixed_zfold_kernel");
        return NEFCT_OK;
    }
    dim3 grid((g->grid.nx + 31) / 32, (g->grid.ny + 31) / 32, g->grid.nz);
    fixed_fold_kernel<<<grid, dim3(32, 8), 0, s>>>(accN, accT, g->grid.nx, g->grid.ny, scale, vol);
    NEFCT_CHECK_LAUNCH("fixed_fold_kernel");
    return NEFCT_OK;
}

template <typename T>
static nefct_status cb_backward_impl(const nefct_cb_geom *g, const T *sino, T *vol, uint32_t flags, void *ws,
                                     size_t wsb, cudaStream_t s)
{
    nefct_status st = check_cb_geom(g);
    if (st) return st;
    if (!vol || !sino) return fail(NEFCT_ERR_INVALID, "vol and sino must be non-NULL");
    if ((st = check_cb_flags(flags))) return st;
    if (flags & NEFCT_DETERMINISTIC) {
        if (sizeof(T) != sizeof(float))
            return fail(NEFCT_ERR_UNSUPPORTED, "NEFCT_DETERMINISTIC is available for float32 only");
        return cb_backward_fixed_impl(g, (const float *)sino, (float *)vol, flags, ws, wsb, s);
    }
    const size_t nvox = (size_t)g->grid.nx * g->grid.ny * g->grid.nz;
    const bool tr = !(flags & NEFCT_NO_TRANSPOSE);
    if (tr && (!ws || wsb < nvox * sizeof(T)))
        return fail(NEFCT_ERR_WORKSPACE, "backward needs %zu workspace bytes, got %zu", nvox * sizeof(T), wsb);
    CBParams<T> *p = new CBParams<T>();
    fill_cb_params(*p, g, flags);
    p->sino = sino;
    p->out = vol;
    p->outT = tr ? (T *)ws : nullptr;
    // column warps reduce into the z-fastest workspace only; the fold then
    // writes every voxel of vol
    const bool cw = cb_use_colwarp<T>(g->grid, flags, false);
    cudaError_t e = cw ? cudaSuccess : cudaMemsetAsync(vol, 0, nvox * sizeof(T), s);
    if (e == cudaSuccess && tr) e = cudaMemsetAsync(ws, 0, nvox * sizeof(T), s);
    if (e != cudaSuccess) { delete p; return cuda_fail(e, "cudaMemsetAsync"); }
    const int kMax = ViewTable<T>::kMax;
    for (int v0 = 0; v0 < g->nv; v0 += kMax) {
        const int nvc = std::min(kMax, g->nv - v0);
        fill_views(*p, g, v0, nvc);
        e = cb_launch_backward<T>(*p, g->na, g->nb, nvc, flags, s, cw);
        if (e != cudaSuccess) { delete p; return cuda_fail(e, "cb_backward_kernel"); }
    }
    delete p;
    if constexpr (std::is_same<T, float>::value) {
        if (cw) return zfold(ws ? (const float *)ws : nullptr, vol, g->grid, s);
    }
    if (tr) {
        dim3 grid((g->grid.nx + 31) / 32, (g->grid.ny + 31) / 32, g->grid.nz);
        fold_add_kernel<T><<<grid, dim3(32, 8), 0, s>>>((const T *)ws, vol, g->grid.nx, g->grid.ny);
        NEFCT_CHECK_LAUNCH("fold_add_kernel");
    }
    return NEFCT_OK;
}

template <typename T>
static nefct_status lor_impl(const nefct_grid *grid, const T *lors, int64_t n, const T *src, T *dst,
                             uint32_t flags, cudaStream_t s, bool forward, const int32_t *order = nullptr)
{
    if (!grid) return fail(NEFCT_ERR_INVALID, "grid is NULL");
    nefct_status st = check_grid(*grid);
    if (st) return st;
    if (n < 0) return fail(NEFCT_ERR_INVALID, "negative LOR count");
    if (flags & (NEFCT_EXACT | NEFCT_DETERMINISTIC | NEFCT_Q8_INDEX))
        return fail(NEFCT_ERR_UNSUPPORTED, "the LOR projector takes the walk flags of cpp/siddon only");
    if ((!lors || !src || !dst) && n > 0) return fail(NEFCT_ERR_INVALID, "NULL buffer");
    if (flags & ~kWalkFlags) return fail(NEFCT_ERR_INVALID, "unknown flag bits 0x%x", flags & ~kWalkFlags);
    if (forward && n == 0) return NEFCT_OK;          // no lines: nothing to write
    if (!dst) return fail(NEFCT_ERR_INVALID, "NULL output");
    LorParams<T> p;
    p.g = make_grid_dev<T>(*grid);
    p.lors = lors; p.n = n; p.flags = flags; p.order = order;
    if (n >= (1ll << 31) && order) return fail(NEFCT_ERR_INVALID, "ordered walks take fewer than 2^31 lines");
    if (!forward) {
        const size_t nvox = (size_t)grid->nx * grid->ny * grid->nz;
        NEFCT_CHECK_CUDA(cudaMemsetAsync(dst, 0, nvox * sizeof(T), s));
        p.vals = src; p.out = dst; p.vol = nullptr;
    } else {
        p.vol = src; p.out = dst; p.vals = nullptr;
    }
    if (n == 0) return NEFCT_OK;
    const long long blocks = std::min<long long>((n + 255) / 256, 148ll * 64);
    const bool q5 = (flags & NEFCT_Q5) != 0, cub = cubic(p.g);
#define NEFCT_LOR_LAUNCH(K)                                                              \
    do {                                                                                 \
        if (cub && !q5) K<T, false, false><<<(unsigned)blocks, 256, 0, s>>>(p);          \
        else if (cub) K<T, false, true><<<(unsigned)blocks, 256, 0, s>>>(p);             \
        else if (!q5) K<T, true, false><<<(unsigned)blocks, 256, 0, s>>>(p);             \
        else K<T, true, true><<<(unsigned)blocks, 256, 0, s>>>(p);                       \
    } while (0)
    if (forward) NEFCT_LOR_LAUNCH(lor_forward_kernel);
    else NEFCT_LOR_LAUNCH(lor_backward_kernel);
#undef NEFCT_LOR_LAUNCH
    NEFCT_CHECK_LAUNCH(forward ? "lor_forward_kernel" : "lor_backward_kernel");
    return NEFCT_OK;
}


// ---------------- forward projection for callers that cannot allocate ----------------
//
// Some callers of this library are not allowed to allocate device memory:
// reconstruction services that reserve all GPU memory at start-up and forbid
// later allocations (fixed memory budget, predictable latency), host
// frameworks that own the device memory pool and only hand out the tensors a
// plugin reads and writes, and bindings that receive bare device pointers
// with no access to an allocator.  nefct_cb_forward needs a volume-sized
// scratch buffer that such callers cannot provide.  For them the scratch
// lives in this fixed array, part of the library's device image: every GPU
// that loads the library holds it (32 MiB) until the process exits.
static constexpr size_t kStaticScratchFloats = size_t(8) << 20;   // 8 Mi voxels
static __device__ __align__(256) float g_static_scratch[kStaticScratchFloats];

// Host code cannot use g_static_scratch's name as a device address.  The
// address belongs to the CUDA context the library's device code is loaded
// in, so it is cached per context, keyed by the context's unique ID
// (cuCtxGetId: never reused within a process), and looked up again
// (cudaGetSymbolAddress) for a context not seen before: the first call in a
// process, on another device, under a caller's own driver-API context, or
// after cudaDeviceReset replaced the device's primary context.  The driver
// calls are reached through cudaGetDriverEntryPoint (no link to libcuda).
using CtxGetCurrentFn = int (*)(void **ctx);
using CtxGetIdFn = int (*)(void *ctx, unsigned long long *id);
static constexpr int kMaxContexts = 64;
static std::mutex g_static_mu;
static CtxGetCurrentFn g_ctx_get_current = nullptr;
static CtxGetIdFn g_ctx_get_id = nullptr;
static unsigned long long g_static_ctx[kMaxContexts];
static float *g_static_addr[kMaxContexts];
static int g_static_n = 0, g_static_next = 0;

// ID of the context current on this thread (have = false: none is current).
// Call with g_static_mu held.
static nefct_status current_context_id(bool &have, unsigned long long &id)
{
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDriverEntryPoint(cuCtxGetCurrent)");
        e = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDriverEntryPoint(cuCtxGetId)");
        if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
            return fail(NEFCT_ERR_UNSUPPORTED, "the driver lacks cuCtxGetCurrent / cuCtxGetId (CUDA 12.0+ needed)");
        g_ctx_get_current = (CtxGetCurrentFn)f1;
        g_ctx_get_id = (CtxGetIdFn)f2;
    }
    void *ctx = nullptr;
    if (g_ctx_get_current(&ctx) != 0) return fail(NEFCT_ERR_CUDA, "cuCtxGetCurrent failed");
    have = ctx != nullptr;
    if (have && g_ctx_get_id(ctx, &id) != 0) return fail(NEFCT_ERR_CUDA, "cuCtxGetId failed");
    return NEFCT_OK;
}

static nefct_status static_scratch_address(float **addr)
{
    std::lock_guard<std::mutex> lock(g_static_mu);
    bool have = false;
    unsigned long long id = 0;
    nefct_status st = current_context_id(have, id);
    if (st) return st;
    if (have) {
        for (int i = 0; i < g_static_n; ++i)
            if (g_static_ctx[i] == id) {
                *addr = g_static_addr[i];
                return NEFCT_OK;
            }
    }
    // a context not seen yet (or none current: the lookup initialises the
    // device's primary context and makes it current)
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_scratch)");
    if (!have) {
        st = current_context_id(have, id);
        if (st) return st;
        if (!have) return fail(NEFCT_ERR_CUDA, "no CUDA context is current after cudaGetSymbolAddress");
    }
    int slot = -1;
    for (int i = 0; i < g_static_n; ++i)
        if (g_static_ctx[i] == id) slot = i;
    if (slot < 0) {
        slot = g_static_n < kMaxContexts ? g_static_n++ : g_static_next;
        g_static_next = (g_static_next + 1) % kMaxContexts;
    }
    g_static_ctx[slot] = id;
    g_static_addr[slot] = (float *)p;
    *addr = (float *)p;
    return NEFCT_OK;
}

static nefct_status cb_forward_static_impl(const nefct_cb_geom *g, const float *vol, float *sino, uint32_t flags,
                                           cudaStream_t s)
{
    nefct_status st = check_cb_geom(g);
    if (st) return st;
    if (!vol || !sino) return fail(NEFCT_ERR_INVALID, "vol and sino must be non-NULL");
    if ((st = check_cb_flags(flags))) return st;
    const size_t nvox = (size_t)g->grid.nx * g->grid.ny * g->grid.nz;
    const bool tr = !(flags & NEFCT_NO_TRANSPOSE);
    if (tr && nvox > kStaticScratchFloats)
        return fail(NEFCT_ERR_INVALID,
                    "nefct_cb_forward_noalloc handles at most %zu voxels (its fixed scratch is %zu MiB); this grid "
                    "has %zu -- use nefct_cb_forward with a workspace",
                    kStaticScratchFloats, kStaticScratchFloats * sizeof(float) >> 20, nvox);
    // the walk nefct_cb_forward takes for these flags and the current
    // launch tuning, over the same kind of volume copy, so the two give the
    // same bits
    const bool cw = cb_use_colwarp<float>(g->grid, flags, true);
    float *scratch = nullptr;
    if (tr) {
        st = static_scratch_address(&scratch);
        if (st) return st;
        // the copy overwrites every scratch element this call reads
        st = cw ? zmajor_copy(vol, scratch, g->grid, s) : transpose_xy(vol, scratch, g->grid, s);
        if (st) return st;
    }
    CBParams<float> p;            // on the host stack: no allocation of any kind
    fill_cb_params(p, g, flags);
    p.vol = vol;
    p.volT = scratch;
    p.out = sino;
    for (int v0 = 0; v0 < g->nv; v0 += ViewTable<float>::kMax) {
        const int nvc = std::min(ViewTable<float>::kMax, g->nv - v0);
        fill_views(p, g, v0, nvc);
        const cudaError_t e = cb_launch_forward<float>(p, g->na, g->nb, nvc, flags, s, cw);
        if (e != cudaSuccess) return cuda_fail(e, "cb_forward_kernel (noalloc)");
    }
    return NEFCT_OK;
}

}  // namespace nefct

using namespace nefct;

extern "C" {

size_t nefct_cb_workspace_bytes(const nefct_cb_geom *g, uint32_t flags)
{
    if (!g || g->grid.nx < 1 || g->grid.ny < 1 || g->grid.nz < 1) return 0;
    if (flags & NEFCT_DETERMINISTIC) return cb_fixed_workspace(g, flags);
    if (flags & NEFCT_NO_TRANSPOSE) return 0;
    return (size_t)(g->grid.nx > 0 ? g->grid.nx : 0) * (size_t)(g->grid.ny > 0 ? g->grid.ny : 0) *
           (size_t)(g->grid.nz > 0 ? g->grid.nz : 0) * sizeof(float);
}

nefct_status nefct_cb_forward(const nefct_cb_geom *g, const float *vol, float *sino, uint32_t flags,
                              void *ws, size_t wsb, void *stream)
{
    return cb_forward_impl<float>(g, vol, sino, flags, ws, wsb, (cudaStream_t)stream);
}

nefct_status nefct_cb_backward(const nefct_cb_geom *g, const float *sino, float *vol, uint32_t flags,
                               void *ws, size_t wsb, void *stream)
{
    return cb_backward_impl<float>(g, sino, vol, flags, ws, wsb, (cudaStream_t)stream);
}

nefct_status nefct_cb_forward_f64(const nefct_cb_geom *g, const double *vol, double *sino, uint32_t flags,
                                  void *ws, size_t wsb, void *stream)
{
    return cb_forward_impl<double>(g, vol, sino, flags, ws, wsb, (cudaStream_t)stream);
}

nefct_status nefct_cb_backward_f64(const nefct_cb_geom *g, const double *sino, double *vol, uint32_t flags,
                                   void *ws, size_t wsb, void *stream)
{
    return cb_backward_impl<double>(g, sino, vol, flags, ws, wsb, (cudaStream_t)stream);
}

nefct_status nefct_cb_count_intersections(const nefct_cb_geom *g, uint32_t flags, unsigned long long *count,
                                          void *stream)
{
    nefct_status st = check_cb_geom(g);
    if (st) return st;
    if (!count) return fail(NEFCT_ERR_INVALID, "count is NULL");
    if (flags & ~kWalkFlags) return fail(NEFCT_ERR_INVALID, "unknown flag bits 0x%x", flags & ~kWalkFlags);
    CBParams<float> *p = new CBParams<float>();
    fill_cb_params(*p, g, flags);
    p->count = count;
    const int kMax = ViewTable<float>::kMax;
    for (int v0 = 0; v0 < g->nv; v0 += kMax) {
        const int nvc = std::min(kMax, g->nv - v0);
        fill_views(*p, g, v0, nvc);
        dim3 grid, block;
        cb_shape(*p, g->na, g->nb, nvc, grid, block);
        if (cubic(p->g)) cb_count_kernel<false><<<grid, block, 0, (cudaStream_t)stream>>>(*p);
        else cb_count_kernel<true><<<grid, block, 0, (cudaStream_t)stream>>>(*p);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { delete p; return cuda_fail(e, "cb_count_kernel"); }
    }
    delete p;
    return NEFCT_OK;
}

nefct_status nefct_lor_forward(const nefct_grid *grid, const float *lors, int64_t n, const float *vol,
                               float *out, uint32_t flags, void *stream)
{
    return lor_impl<float>(grid, lors, n, vol, out, flags, (cudaStream_t)stream, true);
}

nefct_status nefct_lor_backward(const nefct_grid *grid, const float *lors, int64_t n, const float *vals,
                                float *vol, uint32_t flags, void *stream)
{
    return lor_impl<float>(grid, lors, n, vals, vol, flags, (cudaStream_t)stream, false);
}

nefct_status nefct_lor_order_keys(const nefct_grid *grid, const float *lors, int64_t n, int32_t *keys, void *stream)
{
    if (!grid) return fail(NEFCT_ERR_INVALID, "grid is NULL");
    nefct_status st = check_grid(*grid);
    if (st) return st;
    if (n < 0 || n >= (1ll << 31)) return fail(NEFCT_ERR_INVALID, "line count must be in [0, 2^31)");
    if (n == 0) return NEFCT_OK;
    if (!lors || !keys) return fail(NEFCT_ERR_INVALID, "NULL buffer");
    LorParams<float> p{};
    p.g = make_grid_dev<float>(*grid);
    p.lors = lors;
    p.n = n;
    const long long blocks = std::min<long long>((n + 255) / 256, 148ll * 64);
    lor_key_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(p, keys);
    NEFCT_CHECK_LAUNCH("lor_key_kernel");
    return NEFCT_OK;
}

nefct_status nefct_lor_forward_ordered(const nefct_grid *grid, const float *lors, int64_t n, const int32_t *order,
                                       const float *vol, float *out, uint32_t flags, void *stream)
{
    if (!order && n > 0) return fail(NEFCT_ERR_INVALID, "order is NULL");
    return lor_impl<float>(grid, lors, n, vol, out, flags, (cudaStream_t)stream, true, order);
}

nefct_status nefct_lor_backward_ordered(const nefct_grid *grid, const float *lors, int64_t n, const int32_t *order,
                                        const float *vals, float *vol, uint32_t flags, void *stream)
{
    if (!order && n > 0) return fail(NEFCT_ERR_INVALID, "order is NULL");
    return lor_impl<float>(grid, lors, n, vals, vol, flags, (cudaStream_t)stream, false, order);
}

// See cb_forward_static_impl: the same kernels and result as
// nefct_cb_forward, with the scratch in the library's fixed device array
// instead of a caller workspace.
nefct_status nefct_cb_forward_noalloc(const nefct_cb_geom *g, const float *vol, float *sino, uint32_t flags,
                                      void *stream)
{
    return cb_forward_static_impl(g, vol, sino, flags, (cudaStream_t)stream);
}

}  // extern "C"
