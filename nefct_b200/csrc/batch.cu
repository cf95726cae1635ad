// Batched cone-beam problems of uneven sizes.
//
// Two strategies, picked per plan (nefct_cb_batch_set_strategy; the python
// BatchProjector times both):
//  * persistent -- every problem's tiles in one persistent launch per
//    direction (described below);
//  * per-problem -- the single-problem kernels launched once per problem.
// The persistent kernel indexes its problem descriptor dynamically, so the
// per-problem constants that the single-problem kernels read as
// constant-bank operands need registers (the column-warp variant is bounded
// to 64 and spills a little); it pays off when problems are too small to
// fill the GPU one at a time.
//
// A plan holds, for n problems (each with its own grid, views, detector and
// scanner), a table of work tiles -- 32 detector columns x R rows of one
// view for the thread walk, R columns x 32 rows for column warps (the walk
// is fixed at plan time from NEFCT_TUNE_CB_WALK: column warps when both
// directions use them) -- ordered longest rays first (problems sorted by
// slab count, views and row bands inside).  The persistent kernel runs one CTA per resident
// slot; each CTA takes the next tile from an atomic ticket counter until the
// table is exhausted.  Tickets never wait on anything, so the kernel cannot
// hang; load balance across uneven problems comes from the dynamic dequeue
// and the longest-first order.  Forward and transpose are each one
// persistent launch plus the volume copies / folds (with column warps: one
// launch over all problems' tiles, and one memset of all accumulators, which
// are contiguous in the workspace); all work is stream-ordered and
// capturable in a CUDA graph after nefct_cb_batch_bind.
//
// Device workspace (caller-owned), 256-byte aligned sections:
//   counters[4] | view tables | per-problem volume copy
// (problem descriptors and tile offsets travel as kernel parameters)
// The copy (y-fastest for the thread walk, z-fastest for column warps)
// holds the transposed volume during the forward and the accumulator during
// the transpose.
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "cb_kernels.cuh"

namespace nefct {

nefct_status check_cb_geom(const nefct_cb_geom *g);
nefct_status cb_forward_launches(const nefct_cb_geom *g, const float *vol, const float *volT, float *sino,
                                 uint32_t flags, cudaStream_t s, bool colwarp);
nefct_status cb_backward_launches(const nefct_cb_geom *g, const float *sino, float *out, float *outT,
                                  uint32_t flags, cudaStream_t s, bool colwarp);
nefct_status zmajor_copy(const float *in, float *out, const nefct_grid &g, cudaStream_t s);
nefct_status zfold(const float *acc, float *vol, const nefct_grid &g, cudaStream_t s);

struct BatchDesc {
    GridDev<float> g;
    RayGeom<float> rg;
    int na, nb, nv, tiles_a, tiles_b, cubic;
    uint32_t flags;
    const float *cs, *sn, *off;          // per-view tables in the workspace
    const float *vol;
    float *sino;
    const float *grad;
    float *back;
    float *volT;                         // y- or z-fastest copy / accumulator
};

// Descriptors and tile offsets travel in the kernel parameter space (read
// through the constant cache, like the single-problem kernels' parameters),
// which bounds the problems per plan.
static constexpr int kMaxBatch = 96;
struct BatchArgs {
    BatchDesc d[kMaxBatch];
    long long t0[kMaxBatch + 1];
    long long c0[kMaxBatch + 1];         // offsets of the problems' 32 x 32 copy tiles (column warps)
    int n;
    long long begin, end;
    unsigned long long *counter;
};

struct BatchPlan {
    std::vector<nefct_cb_problem> probs;   // caller order; geom.angles/z_offsets point into the copies below
    std::vector<std::vector<float>> angles, offsets;
    int strategy = NEFCT_BATCH_PER_PROBLEM;
    bool colwarp = false;                  // column warps (fixed at plan time)
    std::vector<int> order;                // plan order -> caller index
    std::vector<BatchDesc> desc;           // plan order (device pointers filled at bind)
    std::vector<long long> t0;             // tile offsets, n + 1
    std::vector<long long> c0;             // copy-tile offsets, n + 1 (z-fastest copies and folds)
    std::vector<float> views;              // cs | sn | off per problem, plan order
    std::vector<size_t> view_off, vol_off; // float offsets in the workspace sections
    uint32_t flags = 0;
    int rows = 4;
    long long split = 0;                   // tiles of cubic-voxel problems come first
    size_t off_desc = 0, off_t0 = 0, off_views = 0, off_vols = 0, bytes = 0;
    unsigned char *ws = nullptr;           // bound workspace
    int grid_blocks = 0;
    BatchArgs *args = nullptr;             // launch parameters (host copy)
    ~BatchPlan() { delete args; }
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Tile `item` of the plan -> its problem (largest p with t0[p] <= item).
__device__ __forceinline__ int find_problem(const long long *t0, int n, long long item)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t0[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The z-fastest copies (FOLD false: vol[z][y][x] -> volT[y][x][z]) or folds
// (FOLD true: volT -> back[z][y][x]) of every problem in one launch: the
// 32 x 32 (x, z) tiles of all problems' y planes, tile t of problem p at
// c0[p] + ((y * tiles_z) + tz) * tiles_x + tx, grid-strided.
template <bool FOLD>
__global__ void __launch_bounds__(256) batch_zcopy_kernel(const __grid_constant__ BatchArgs a, long long total)
{
    __shared__ float tile[32][33];
    for (long long t = blockIdx.x; t < total; t += gridDim.x) {     // uniform across the CTA
        const int p = find_problem(a.c0, a.n, t);
        const BatchDesc &P = a.d[p];
        const int nx = P.g.nx, ny = P.g.ny, nz = P.g.nz;
        const int tiles_x = (nx + 31) / 32, tiles_z = (nz + 31) / 32;
        const long long local = t - a.c0[p];
        const int x0 = (int)(local % tiles_x) * 32;
        const long long rest = local / tiles_x;
        const int z0 = (int)(rest % tiles_z) * 32;
        const int y = (int)(rest / tiles_z);
        if (!FOLD) {
            for (int j = threadIdx.y; j < 32; j += 8) {
                const int x = x0 + threadIdx.x, z = z0 + j;
                if (x < nx && z < nz) tile[j][threadIdx.x] = P.vol[((size_t)z * ny + y) * nx + x];
            }
            __syncthreads();
            for (int j = threadIdx.y; j < 32; j += 8) {
                const int x = x0 + j, z = z0 + threadIdx.x;
                if (x < nx && z < nz) P.volT[((size_t)y * nx + x) * nz + z] = tile[threadIdx.x][j];
            }
        } else {
            for (int j = threadIdx.y; j < 32; j += 8) {
                const int x = x0 + j, z = z0 + threadIdx.x;
                if (x < nx && z < nz) tile[j][threadIdx.x] = P.volT[((size_t)y * nx + x) * nz + z];
            }
            __syncthreads();
            for (int j = threadIdx.y; j < 32; j += 8) {
                const int x = x0 + threadIdx.x, z = z0 + j;
                if (x < nx && z < nz) P.back[((size_t)z * ny + y) * nx + x] = tile[threadIdx.x][j];
            }
        }
        __syncthreads();                  // the tile is read before the next iteration rewrites it
    }
}

// One persistent launch serves tiles [begin, end) of problems that share
// the DIV variant (cubic voxels or not).
template <bool FWD, bool DIV>
__global__ void __launch_bounds__(256) batch_kernel(const __grid_constant__ BatchArgs a)
{
    __shared__ long long s_item;
    for (;;) {
        if (threadIdx.x == 0 && threadIdx.y == 0) s_item = a.begin + (long long)atomicAdd(a.counter, 1ull);
        __syncthreads();
        const long long item = s_item;
        __syncthreads();                  // all threads read s_item before the next ticket
        if (item >= a.end) return;        // uniform across the CTA
        const int p = find_problem(a.t0, a.n, item);
        const BatchDesc &P = a.d[p];
        const long long local = item - a.t0[p];
        const int ct = (int)(local % P.tiles_a);
        const long long rest = local / P.tiles_a;
        const int band = (int)(rest % P.tiles_b);
        const int iv = (int)(rest / P.tiles_b);
        const int ia = ct * 32 + threadIdx.x, ib = band * blockDim.y + threadIdx.y;
        if (ia >= P.na || ib >= P.nb) continue;
        float r[6];
        cb_ray(P.rg, P.cs[iv], P.sn[iv], P.off[iv], ia, ib, r);
        const size_t id = ((size_t)iv * P.nb + ib) * P.na + ia;
        if (FWD) {
            P.sino[id] = ray_forward<float, DIV>(P.g, r, P.flags, P.vol, P.volT);
        } else {
            const float y = P.grad[id];
            if (y == 0.f) continue;
            ray_backward<float, DIV>(P.g, r, P.flags, y, P.back, P.volT);
        }
    }
}

// Column-warp variant: a tile is blockDim.y columns x 32 rows of one view,
// one warp per column.  Bounded to 64 registers (4 CTAs of 256 threads per
// SM) like the single-problem kernels: the dynamically indexed problem
// descriptor then spills 100-260 bytes, and the kernel still runs faster
// than at its unbounded 80-94 registers (96 small problems: 4.67 against
// 5.26 ms per forward + transpose).
template <bool FWD, bool DIV>
__global__ void __launch_bounds__(256, 4) batch_colwarp_kernel(const __grid_constant__ BatchArgs a)
{
    __shared__ long long s_item;
    for (;;) {
        if (threadIdx.x == 0 && threadIdx.y == 0) s_item = a.begin + (long long)atomicAdd(a.counter, 1ull);
        __syncthreads();
        const long long item = s_item;
        __syncthreads();                  // all threads read s_item before the next ticket
        if (item >= a.end) return;        // uniform across the CTA
        const int p = find_problem(a.t0, a.n, item);
        const BatchDesc &P = a.d[p];
        const long long local = item - a.t0[p];
        const int ct = (int)(local % P.tiles_a);
        const long long rest = local / P.tiles_a;
        const int rt = (int)(rest % P.tiles_b);
        const int iv = (int)(rest / P.tiles_b);
        const int ia = ct * blockDim.y + threadIdx.y, ib = rt * 32 + threadIdx.x;
        if (ia >= P.na) continue;         // uniform across the warp
        const bool has = ib < P.nb;
        const size_t id = ((size_t)iv * P.nb + (has ? ib : 0)) * P.na + ia;
        float r[6];
        cb_ray(P.rg, P.cs[iv], P.sn[iv], P.off[iv], ia, has ? ib : 0, r);
        if (FWD) colwarp_lane<DIV, true>(P.g, r, has, P.flags, P.volT, P.sino + id, 0.f, nullptr);
        else colwarp_lane<DIV, false>(P.g, r, has, P.flags, nullptr, nullptr, has ? P.grad[id] : 0.f, P.volT);
    }
}

// Per-problem strategy: the single-problem kernels launched once per problem
// (their scanner constants as kernel parameters), stream-ordered.
static nefct_status batch_per_problem(BatchPlan *b, bool fwd, cudaStream_t s)
{
    const int n = (int)b->desc.size();
    for (int k = 0; k < n; ++k) {
        const BatchDesc &D = b->desc[k];
        const nefct_cb_geom &g = b->probs[b->order[k]].geom;
        const size_t nvox = (size_t)D.g.nx * D.g.ny * D.g.nz;
        dim3 tg((D.g.nx + 31) / 32, (D.g.ny + 31) / 32, D.g.nz);
        nefct_status st;
        if (b->colwarp) {
            if (fwd) {
                st = zmajor_copy(D.vol, D.volT, g.grid, s);
                if (!st) st = cb_forward_launches(&g, D.vol, D.volT, D.sino, D.flags, s, true);
            } else {
                NEFCT_CHECK_CUDA(cudaMemsetAsync(D.volT, 0, nvox * sizeof(float), s));
                st = cb_backward_launches(&g, D.grad, D.back, D.volT, D.flags, s, true);
                if (!st) st = zfold(D.volT, D.back, g.grid, s);
            }
        } else if (fwd) {
            transpose_xy_kernel<float><<<tg, dim3(32, 8), 0, s>>>(D.vol, D.volT, D.g.nx, D.g.ny);
            NEFCT_CHECK_LAUNCH("transpose_xy_kernel (batch)");
            st = cb_forward_launches(&g, D.vol, D.volT, D.sino, D.flags, s, false);
        } else {
            NEFCT_CHECK_CUDA(cudaMemsetAsync(D.back, 0, nvox * sizeof(float), s));
            NEFCT_CHECK_CUDA(cudaMemsetAsync(D.volT, 0, nvox * sizeof(float), s));
            st = cb_backward_launches(&g, D.grad, D.back, D.volT, D.flags, s, false);
            if (!st) {
                fold_add_kernel<float><<<tg, dim3(32, 8), 0, s>>>(D.volT, D.back, D.g.nx, D.g.ny);
                NEFCT_CHECK_LAUNCH("fold_add_kernel (batch)");
            }
        }
        if (st) return st;
    }
    return NEFCT_OK;
}

static nefct_status batch_launch(BatchPlan *b, bool fwd, cudaStream_t s)
{
    if (!b || !b->ws) return fail(NEFCT_ERR_INVALID, "batch plan is not bound to a workspace");
    if (b->strategy == NEFCT_BATCH_PER_PROBLEM) return batch_per_problem(b, fwd, s);
    const int n = (int)b->desc.size();
    unsigned long long *counter = (unsigned long long *)b->ws + (fwd ? 0 : 2);
    NEFCT_CHECK_CUDA(cudaMemsetAsync(counter, 0, 2 * sizeof(unsigned long long), s));
    BatchArgs &ca = *b->args;
    const long long copy_tiles = b->c0.back();
    const unsigned copy_blocks = (unsigned)std::min<long long>(copy_tiles, 148ll * 8);
    if (b->colwarp) {
        // one launch for all problems' z-fastest copies (forward) or one memset
        // of every accumulator (transpose; they are contiguous in the workspace)
        if (fwd) {
            batch_zcopy_kernel<false><<<copy_blocks, dim3(32, 8), 0, s>>>(ca, copy_tiles);
            NEFCT_CHECK_LAUNCH("batch_zcopy_kernel");
        } else {
            NEFCT_CHECK_CUDA(cudaMemsetAsync(b->ws + b->off_vols, 0, b->bytes - b->off_vols, s));
        }
    }
    for (int i = 0; i < n && !b->colwarp; ++i) {
        const BatchDesc &D = b->desc[i];
        const size_t nvox = (size_t)D.g.nx * D.g.ny * D.g.nz;
        dim3 tg((D.g.nx + 31) / 32, (D.g.ny + 31) / 32, D.g.nz);
        if (fwd) {
            transpose_xy_kernel<float><<<tg, dim3(32, 8), 0, s>>>(D.vol, D.volT, D.g.nx, D.g.ny);
            NEFCT_CHECK_LAUNCH("transpose_xy_kernel (batch)");
        } else {
            NEFCT_CHECK_CUDA(cudaMemsetAsync(D.back, 0, nvox * sizeof(float), s));
            NEFCT_CHECK_CUDA(cudaMemsetAsync(D.volT, 0, nvox * sizeof(float), s));
        }
    }
    const long long total = b->t0.back();
    const dim3 blk(32, b->rows);
    BatchArgs &a = *b->args;
    if (b->split > 0) {
        a.begin = 0; a.end = b->split; a.counter = counter;
        if (b->colwarp) {
            if (fwd) batch_colwarp_kernel<true, false><<<b->grid_blocks, blk, 0, s>>>(a);
            else batch_colwarp_kernel<false, false><<<b->grid_blocks, blk, 0, s>>>(a);
        } else {
            if (fwd) batch_kernel<true, false><<<b->grid_blocks, blk, 0, s>>>(a);
            else batch_kernel<false, false><<<b->grid_blocks, blk, 0, s>>>(a);
        }
        NEFCT_CHECK_LAUNCH("batch_kernel (cubic voxels)");
    }
    if (b->split < total) {
        a.begin = b->split; a.end = total; a.counter = counter + 1;
        if (b->colwarp) {
            if (fwd) batch_colwarp_kernel<true, true><<<b->grid_blocks, blk, 0, s>>>(a);
            else batch_colwarp_kernel<false, true><<<b->grid_blocks, blk, 0, s>>>(a);
        } else {
            if (fwd) batch_kernel<true, true><<<b->grid_blocks, blk, 0, s>>>(a);
            else batch_kernel<false, true><<<b->grid_blocks, blk, 0, s>>>(a);
        }
        NEFCT_CHECK_LAUNCH("batch_kernel (other voxels)");
    }
    if (!fwd && b->colwarp) {
        batch_zcopy_kernel<true><<<copy_blocks, dim3(32, 8), 0, s>>>(ca, copy_tiles);
        NEFCT_CHECK_LAUNCH("batch_zcopy_kernel (fold)");
    } else if (!fwd) {
        for (int i = 0; i < n; ++i) {
            const BatchDesc &D = b->desc[i];
            dim3 tg((D.g.nx + 31) / 32, (D.g.ny + 31) / 32, D.g.nz);
            fold_add_kernel<float><<<tg, dim3(32, 8), 0, s>>>(D.volT, D.back, D.g.nx, D.g.ny);
            NEFCT_CHECK_LAUNCH("fold_add_kernel (batch)");
        }
    }
    return NEFCT_OK;
}

}  // namespace nefct

using namespace nefct;

struct nefct_cb_batch : BatchPlan {};

extern "C" {

nefct_status nefct_cb_batch_plan(const nefct_cb_problem *problems, int32_t n, uint32_t flags,
                                 nefct_cb_batch **plan, size_t *workspace_bytes)
{
    if (!plan || !workspace_bytes) return fail(NEFCT_ERR_INVALID, "plan and workspace_bytes must be non-NULL");
    *plan = nullptr;
    if (n < 1 || !problems) return fail(NEFCT_ERR_INVALID, "need at least one problem");
    if (n > kMaxBatch) return fail(NEFCT_ERR_INVALID, "at most %d problems per batch plan (got %d)", kMaxBatch, n);
    if (flags & ~(NEFCT_TIE_GT | NEFCT_SKIP_SHORT | NEFCT_NO_INV_L2))
        return fail(NEFCT_ERR_INVALID, "flags 0x%x not supported by the batch", flags);
    for (int i = 0; i < n; ++i) {
        nefct_status st = check_cb_geom(&problems[i].geom);
        if (st) {
            const std::string msg = nefct_last_error();
            return fail(st, "problem %d: %s", i, msg.c_str());
        }
        const nefct_cb_problem &P = problems[i];
        if (!P.vol || !P.sino || !P.grad || !P.back) return fail(NEFCT_ERR_INVALID, "problem %d: NULL buffer", i);
    }
    nefct_cb_batch *b = new nefct_cb_batch();
    b->probs.assign(problems, problems + n);
    b->angles.resize(n);
    b->offsets.resize(n);
    for (int i = 0; i < n; ++i) {
        nefct_cb_geom &g = b->probs[i].geom;
        b->angles[i].assign(g.angles, g.angles + g.nv);
        g.angles = b->angles[i].data();
        if (g.z_offsets) {
            b->offsets[i].assign(g.z_offsets, g.z_offsets + g.nv);
            g.z_offsets = b->offsets[i].data();
        }
    }
    b->flags = flags;
    b->rows = tune_get(NEFCT_TUNE_CB_ROWS);
    b->colwarp = tune_get(NEFCT_TUNE_CB_WALK) == 3;
    for (int i = 0; i < n; ++i)
        b->colwarp = b->colwarp && cb_use_colwarp<float>(problems[i].geom.grid, flags, true) &&
                     cb_use_colwarp<float>(problems[i].geom.grid, flags, false);
    // cubic-voxel problems first (one kernel variant each), longest rays
    // first within each group: a tile's cost grows with its rays' slab count
    auto cubic = [&](int i) {
        const GridDev<float> g = make_grid_dev<float>(problems[i].geom.grid);
        return g.dy == 1.f && g.dz == 1.f;
    };
    b->order.resize(n);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int c) {
        const bool ca = cubic(a), cc = cubic(c);
        if (ca != cc) return ca;
        const nefct_grid &ga = problems[a].geom.grid, &gc = problems[c].geom.grid;
        return std::max(ga.nx, ga.ny) > std::max(gc.nx, gc.ny);
    });
    b->desc.resize(n);
    b->t0.assign(n + 1, 0);
    b->c0.assign(n + 1, 0);
    size_t views = 0, vols = 0;
    b->view_off.resize(n);
    b->vol_off.resize(n);
    for (int k = 0; k < n; ++k) {
        const nefct_cb_geom &g = problems[b->order[k]].geom;
        BatchDesc &D = b->desc[k];
        D.g = make_grid_dev<float>(g.grid);
        D.rg = make_ray_geom<float>(g);
        D.na = g.na; D.nb = g.nb; D.nv = g.nv;
        D.tiles_a = b->colwarp ? (g.na + b->rows - 1) / b->rows : (g.na + 31) / 32;
        D.tiles_b = b->colwarp ? (g.nb + 31) / 32 : (g.nb + b->rows - 1) / b->rows;
        D.cubic = D.g.dy == 1.f && D.g.dz == 1.f;
        D.flags = flags;
        b->t0[k + 1] = b->t0[k] + (long long)D.tiles_a * D.tiles_b * g.nv;
        b->c0[k + 1] = b->c0[k] + (long long)((g.grid.nx + 31) / 32) * ((g.grid.nz + 31) / 32) * g.grid.ny;
        if (D.cubic) b->split = b->t0[k + 1];
        b->view_off[k] = views;
        views += 3 * (size_t)g.nv;
        b->vol_off[k] = vols;
        vols += align256((size_t)g.grid.nx * g.grid.ny * g.grid.nz * sizeof(float)) / sizeof(float);
    }
    b->views.resize(views);
    for (int k = 0; k < n; ++k) {
        const nefct_cb_geom &g = problems[b->order[k]].geom;
        float *v = b->views.data() + b->view_off[k];
        for (int i = 0; i < g.nv; ++i) {
            v[i] = (float)cos((double)g.angles[i]);
            v[g.nv + i] = (float)sin((double)g.angles[i]);
            v[2 * g.nv + i] = g.z_offsets ? g.z_offsets[i] : 0.f;
        }
    }
    b->off_desc = align256(4 * sizeof(unsigned long long));
    b->off_t0 = b->off_desc;
    b->off_views = b->off_desc;
    b->off_vols = b->off_views + align256(views * sizeof(float));
    b->bytes = b->off_vols + vols * sizeof(float);
    *workspace_bytes = b->bytes;
    *plan = b;
    return NEFCT_OK;
}

nefct_status nefct_cb_batch_bind(nefct_cb_batch *b, void *workspace, size_t bytes, void *stream)
{
    if (!b) return fail(NEFCT_ERR_INVALID, "plan is NULL");
    if (!workspace || bytes < b->bytes)
        return fail(NEFCT_ERR_WORKSPACE, "batch needs %zu workspace bytes, got %zu", b->bytes, bytes);
    if ((uintptr_t)workspace & 255) return fail(NEFCT_ERR_INVALID, "workspace must be 256-byte aligned");
    unsigned char *ws = (unsigned char *)workspace;
    const int n = (int)b->desc.size();
    for (int k = 0; k < n; ++k) {
        const nefct_cb_problem &P = b->probs[b->order[k]];
        BatchDesc &D = b->desc[k];
        const float *v = (const float *)(ws + b->off_views) + b->view_off[k];
        D.cs = v; D.sn = v + D.nv; D.off = v + 2 * D.nv;
        D.vol = P.vol; D.sino = P.sino; D.grad = P.grad; D.back = P.back;
        D.volT = (float *)(ws + b->off_vols) + b->vol_off[k];
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->args) b->args = new BatchArgs();
    std::copy(b->desc.begin(), b->desc.end(), b->args->d);
    std::copy(b->t0.begin(), b->t0.end(), b->args->t0);
    std::copy(b->c0.begin(), b->c0.end(), b->args->c0);
    b->args->n = n;
    NEFCT_CHECK_CUDA(cudaMemcpyAsync(ws + b->off_views, b->views.data(), b->views.size() * sizeof(float),
                                     cudaMemcpyHostToDevice, s));
    // the copies read the plan's host memory: finish them before returning
    NEFCT_CHECK_CUDA(cudaStreamSynchronize(s));
    int dev = 0, sms = 0, per_sm = 0;
    NEFCT_CHECK_CUDA(cudaGetDevice(&dev));
    NEFCT_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int lo = 1 << 30;
    const void *kernels[4] = {(const void *)batch_kernel<true, false>, (const void *)batch_kernel<true, true>,
                              (const void *)batch_kernel<false, false>, (const void *)batch_kernel<false, true>};
    const void *colwarp_kernels[4] = {
        (const void *)batch_colwarp_kernel<true, false>, (const void *)batch_colwarp_kernel<true, true>,
        (const void *)batch_colwarp_kernel<false, false>, (const void *)batch_colwarp_kernel<false, true>};
    for (const void *k : b->colwarp ? colwarp_kernels : kernels) {
        NEFCT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * b->rows, 0));
        lo = std::min(lo, per_sm);
    }
    b->grid_blocks = sms * std::max(1, lo);
    b->ws = ws;
    return NEFCT_OK;
}

nefct_status nefct_cb_batch_forward(nefct_cb_batch *b, void *stream)
{
    return batch_launch(b, true, (cudaStream_t)stream);
}

nefct_status nefct_cb_batch_backward(nefct_cb_batch *b, void *stream)
{
    return batch_launch(b, false, (cudaStream_t)stream);
}

int64_t nefct_cb_batch_tiles(const nefct_cb_batch *b) { return b ? (int64_t)b->t0.back() : -1; }

nefct_status nefct_cb_batch_set_strategy(nefct_cb_batch *b, int32_t strategy)
{
    if (!b) return fail(NEFCT_ERR_INVALID, "plan is NULL");
    if (strategy != NEFCT_BATCH_PERSISTENT && strategy != NEFCT_BATCH_PER_PROBLEM)
        return fail(NEFCT_ERR_INVALID, "unknown batch strategy %d", strategy);
    b->strategy = strategy;
    return NEFCT_OK;
}

nefct_status nefct_cb_batch_set_buffers(nefct_cb_batch *b, const float *const *vols, float *const *sinos,
                                        const float *const *grads, float *const *backs)
{
    if (!b) return fail(NEFCT_ERR_INVALID, "plan is NULL");
    const int n = (int)b->desc.size();
    for (int k = 0; k < n; ++k) {
        const int i = b->order[k];
        nefct_cb_problem &P = b->probs[i];
        if (vols && vols[i]) P.vol = vols[i];
        if (sinos && sinos[i]) P.sino = sinos[i];
        if (grads && grads[i]) P.grad = grads[i];
        if (backs && backs[i]) P.back = backs[i];
        BatchDesc &D = b->desc[k];
        D.vol = P.vol; D.sino = P.sino; D.grad = P.grad; D.back = P.back;
        if (b->args) {
            BatchDesc &A = b->args->d[k];
            A.vol = P.vol; A.sino = P.sino; A.grad = P.grad; A.back = P.back;
        }
    }
    return NEFCT_OK;
}

void nefct_cb_batch_destroy(nefct_cb_batch *b) { delete b; }

}  // extern "C"
