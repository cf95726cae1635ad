// Ceiling probes for the projector rooflines (sm_100a).
//
// The cone-beam walks gather (forward) and reduce (transpose) 4-byte values
// that are mostly L2-resident: their binding ceilings are the L2 read
// bandwidth and the L2 reduction rate, not the HBM copy bandwidth.  These
// two kernels measure both on the GPU they run on, over a caller-given
// buffer small enough to stay in L2 (tens of MB):
//  * l2_read_kernel streams the buffer with 16-byte L2-only loads
//    (ld.global.cg, no L1 allocation) `reps` times;
//  * l2_red_kernel issues one red.global.add.f32 per 4-byte element per
//    pass, a warp covering 32 consecutive elements (4 sectors per request),
//    `reps` times.
// Grids are persistent: blocks_per_sm x SM count CTAs of 256 threads.
#include <algorithm>

#include "common.cuh"

namespace nefct {

__global__ void __launch_bounds__(256) l2_read_kernel(const float4 *__restrict__ buf, size_t n4, int reps,
                                                      float *sink)
{
    float acc = 0.f;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; ++r) {
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
            float4 v;
            asm volatile("ld.global.cg.v4.f32 {%0, %1, %2, %3}, [%4];"
                         : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                         : "l"(buf + i));
            acc += (v.x + v.y) + (v.z + v.w);
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sink[blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32] = acc;
}

__global__ void __launch_bounds__(256) l2_red_kernel(float *buf, size_t n, int reps)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; ++r)
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride)
            asm volatile("red.global.add.f32 [%0], %1;" ::"l"(buf + i), "f"(1.0f) : "memory");
}

static nefct_status probe_grid(int blocks_per_sm, unsigned &blocks)
{
    if (blocks_per_sm < 1 || blocks_per_sm > 32) return fail(NEFCT_ERR_INVALID, "blocks_per_sm must be in [1, 32]");
    int dev = 0, sms = 0;
    NEFCT_CHECK_CUDA(cudaGetDevice(&dev));
    NEFCT_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    blocks = (unsigned)(sms * blocks_per_sm);
    return NEFCT_OK;
}

}  // namespace nefct

using namespace nefct;

extern "C" {

size_t nefct_probe_sink_floats(int32_t blocks_per_sm)
{
    unsigned blocks = 0;
    if (probe_grid(blocks_per_sm, blocks) != NEFCT_OK) return 0;
    return (size_t)blocks * 8;
}

nefct_status nefct_probe_l2_read(const float *buf, size_t n, int32_t reps, int32_t blocks_per_sm, float *sink,
                                 void *stream)
{
    if (!buf || !sink) return fail(NEFCT_ERR_INVALID, "buf and sink must be non-NULL");
    if (n < 4 || n % 4 != 0) return fail(NEFCT_ERR_INVALID, "n must be a positive multiple of 4 floats");
    if (((uintptr_t)buf & 15) != 0) return fail(NEFCT_ERR_INVALID, "buf must be 16-byte aligned");
    if (reps < 1) return fail(NEFCT_ERR_INVALID, "reps must be >= 1");
    unsigned blocks = 0;
    nefct_status st = probe_grid(blocks_per_sm, blocks);
    if (st) return st;
    l2_read_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>((const float4 *)buf, n / 4, reps, sink);
    NEFCT_CHECK_LAUNCH("l2_read_kernel");
    return NEFCT_OK;
}

nefct_status nefct_probe_l2_red(float *buf, size_t n, int32_t reps, int32_t blocks_per_sm, void *stream)
{
    if (!buf || n == 0) return fail(NEFCT_ERR_INVALID, "buf must be non-NULL and n > 0");
    if (reps < 1) return fail(NEFCT_ERR_INVALID, "reps must be >= 1");
    unsigned blocks = 0;
    nefct_status st = probe_grid(blocks_per_sm, blocks);
    if (st) return st;
    l2_red_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(buf, n, reps);
    NEFCT_CHECK_LAUNCH("l2_red_kernel");
    return NEFCT_OK;
}

}  // extern "C"
