// Batched cone-beam problems of uneven sizes in one persistent launch.
//
// A plan holds, for n problems (each with its own grid, views, detector and
// scanner), a table of work tiles -- 32 detector columns x R rows of one
// view -- ordered longest rays first (problems sorted by slab count, views
// and row bands inside).  The persistent kernel runs one CTA per resident
// slot; each CTA takes the next tile from an atomic ticket counter until the
// table is exhausted.  Tickets never wait on anything, so the kernel cannot
// hang; load balance across uneven problems comes from the dynamic dequeue
// and the longest-first order.  Forward and transpose are each one
// persistent launch plus per-problem transposes/folds; all work is
// stream-ordered and capturable in a CUDA graph after nefct_cb_batch_bind.
//
// Device workspace (caller-owned), 256-byte aligned sections:
//   counters[2] | descriptors[n] | tile offsets[n+1] | view tables | per-problem y-fastest volume
// The y-fastest copy holds the transposed volume during the forward and
// the accumulator of x-driven rays during the transpose.
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "siddon.cuh"

namespace nefct {

nefct_status check_cb_geom(const nefct_cb_geom *g);

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
    float *volT;                         // y-fastest copy / accumulator
};

struct BatchPlan {
    std::vector<nefct_cb_problem> probs;   // caller order
    std::vector<int> order;                // plan order -> caller index
    std::vector<BatchDesc> desc;           // plan order (device pointers filled at bind)
    std::vector<long long> t0;             // tile offsets, n + 1
    std::vector<float> views;              // cs | sn | off per problem, plan order
    std::vector<size_t> view_off, vol_off; // float offsets in the workspace sections
    uint32_t flags = 0;
    int rows = 4;
    size_t off_desc = 0, off_t0 = 0, off_views = 0, off_vols = 0, bytes = 0;
    unsigned char *ws = nullptr;           // bound workspace
    int grid_blocks = 0;
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Tile `item` of the plan -> (problem, view, first column, first row).
__device__ __forceinline__ int find_problem(const long long *__restrict__ t0, int n, long long item)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t0[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <bool FWD>
__global__ void __launch_bounds__(256) batch_kernel(const BatchDesc *__restrict__ d, const long long *__restrict__ t0,
                                                    int n, unsigned long long *counter)
{
    __shared__ long long s_item;
    const long long total = t0[n];
    for (;;) {
        if (threadIdx.x == 0 && threadIdx.y == 0) s_item = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const long long item = s_item;
        __syncthreads();                  // all threads read s_item before the next ticket
        if (item >= total) return;        // uniform across the CTA
        const int p = find_problem(t0, n, item);
        const BatchDesc &P = d[p];
        const long long local = item - t0[p];
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
            const float acc = P.cubic ? ray_forward<float, false>(P.g, r, P.flags, P.vol, P.volT)
                                      : ray_forward<float, true>(P.g, r, P.flags, P.vol, P.volT);
            P.sino[id] = acc;
        } else {
            const float y = P.grad[id];
            if (y == 0.f) continue;
            if (P.cubic) ray_backward<float, false>(P.g, r, P.flags, y, P.back, P.volT);
            else ray_backward<float, true>(P.g, r, P.flags, y, P.back, P.volT);
        }
    }
}

static nefct_status batch_launch(const BatchPlan *b, bool fwd, cudaStream_t s)
{
    if (!b || !b->ws) return fail(NEFCT_ERR_INVALID, "batch plan is not bound to a workspace");
    const int n = (int)b->desc.size();
    unsigned long long *counter = (unsigned long long *)b->ws + (fwd ? 0 : 1);
    NEFCT_CHECK_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    for (int i = 0; i < n; ++i) {
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
    const BatchDesc *dd = (const BatchDesc *)(b->ws + b->off_desc);
    const long long *t0 = (const long long *)(b->ws + b->off_t0);
    if (fwd) batch_kernel<true><<<b->grid_blocks, dim3(32, b->rows), 0, s>>>(dd, t0, n, counter);
    else batch_kernel<false><<<b->grid_blocks, dim3(32, b->rows), 0, s>>>(dd, t0, n, counter);
    NEFCT_CHECK_LAUNCH("batch_kernel");
    if (!fwd) {
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
    b->flags = flags;
    b->rows = tune_get(NEFCT_TUNE_CB_ROWS);
    // longest rays first: a tile's cost grows with the slab count of its rays
    b->order.resize(n);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int c) {
        const nefct_grid &ga = problems[a].geom.grid, &gc = problems[c].geom.grid;
        return std::max(ga.nx, ga.ny) > std::max(gc.nx, gc.ny);
    });
    b->desc.resize(n);
    b->t0.assign(n + 1, 0);
    size_t views = 0, vols = 0;
    b->view_off.resize(n);
    b->vol_off.resize(n);
    for (int k = 0; k < n; ++k) {
        const nefct_cb_geom &g = problems[b->order[k]].geom;
        BatchDesc &D = b->desc[k];
        D.g = make_grid_dev<float>(g.grid);
        D.rg = make_ray_geom<float>(g);
        D.na = g.na; D.nb = g.nb; D.nv = g.nv;
        D.tiles_a = (g.na + 31) / 32;
        D.tiles_b = (g.nb + b->rows - 1) / b->rows;
        D.cubic = D.g.dy == 1.f && D.g.dz == 1.f;
        D.flags = flags;
        b->t0[k + 1] = b->t0[k] + (long long)D.tiles_a * D.tiles_b * g.nv;
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
    b->off_desc = align256(2 * sizeof(unsigned long long));
    b->off_t0 = b->off_desc + align256(n * sizeof(BatchDesc));
    b->off_views = b->off_t0 + align256((n + 1) * sizeof(long long));
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
    NEFCT_CHECK_CUDA(cudaMemcpyAsync(ws + b->off_desc, b->desc.data(), n * sizeof(BatchDesc), cudaMemcpyHostToDevice, s));
    NEFCT_CHECK_CUDA(cudaMemcpyAsync(ws + b->off_t0, b->t0.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, s));
    NEFCT_CHECK_CUDA(cudaMemcpyAsync(ws + b->off_views, b->views.data(), b->views.size() * sizeof(float),
                                     cudaMemcpyHostToDevice, s));
    // the copies read the plan's host memory: finish them before returning
    NEFCT_CHECK_CUDA(cudaStreamSynchronize(s));
    int dev = 0, sms = 0, per_sm = 0;
    NEFCT_CHECK_CUDA(cudaGetDevice(&dev));
    NEFCT_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    NEFCT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<true>, 32 * b->rows, 0));
    int per_sm_b = 0;
    NEFCT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_b, batch_kernel<false>, 32 * b->rows, 0));
    b->grid_blocks = sms * std::max(1, std::min(per_sm, per_sm_b));
    b->ws = ws;
    return NEFCT_OK;
}

nefct_status nefct_cb_batch_forward(const nefct_cb_batch *b, void *stream)
{
    return batch_launch(b, true, (cudaStream_t)stream);
}

nefct_status nefct_cb_batch_backward(const nefct_cb_batch *b, void *stream)
{
    return batch_launch(b, false, (cudaStream_t)stream);
}

int64_t nefct_cb_batch_tiles(const nefct_cb_batch *b) { return b ? (int64_t)b->t0.back() : -1; }

void nefct_cb_batch_destroy(nefct_cb_batch *b) { delete b; }

}  // extern "C"
