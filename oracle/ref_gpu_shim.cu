// TEST INFRASTRUCTURE: the reference's siddon_3d cone-beam kernels and their
// host launchers (nefct/cc/siddon_3d/siddon.cu.cc:6-890: project_device,
// ProjectFlatKernel, project_flat, backproject_device, BackProjectFlatKernel,
// backproject_flat, ...) built unchanged by nvcc from the reference checkout
// (the Makefile extracts the line range into _ref/gen/siddon3d_gpu.inc).  It
// runs the reference's own CUDA path on the GPU for the parity tests and for
// timing that path beside the library's.  Only tests load it.
//
// The flat-detector kernels index the volume only under their own range
// checks (every image access and atomicAdd sits behind 0 <= c < n tests of
// its indices, and the sinogram index ia + ib*na + iv*na*nb stays below
// na*nb*nv); the cylindrical backprojection's sinogram index (quirk Q8,
// :830) can leave the buffer when nb > nv, so only the flat pair is exported.
#include <cuda_runtime.h>

#include "siddon3d_gpu.inc"

namespace {

struct HostGrid {
    int dims[3];
    float center[3];
    float size[3];
};

// The reference's host functions read grid / center / size back from the
// device (siddon.cu.cc:401-406), so they are staged in one device block.
// Runs on the legacy default stream like the reference and synchronises.
int run(bool forward, const float *in, const HostGrid &hg, const float *angles, int na, int nb, int nv, float SID,
        float SAD, float da, float ai, float db, float bi, float *out)
{
    unsigned char *blk = nullptr;
    cudaError_t e = cudaMalloc(&blk, sizeof(HostGrid));
    if (e != cudaSuccess) return (int)e;
    e = cudaMemcpy(blk, &hg, sizeof(HostGrid), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int *grid = (const int *)blk;
        const float *center = (const float *)(blk + offsetof(HostGrid, center));
        const float *size = (const float *)(blk + offsetof(HostGrid, size));
        if (forward) project_flat(in, grid, center, size, angles, na, nb, nv, SID, SAD, da, ai, db, bi, out);
        else backproject_flat(in, grid, center, size, angles, na, nb, nv, SID, SAD, da, ai, db, bi, out);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    cudaFree(blk);
    return (int)e;
}

}  // namespace

extern "C" {

// vol: device [nz][ny][nx]; angles: device [nv]; sino: device [nv][nb][na].
// Geometry in the reference kernels' naming (SID source-isocentre, SAD
// source-detector).  Returns the CUDA error code (0 = success).
int ref_gpu_project_flat(const float *vol, int nx, int ny, int nz, float cx, float cy, float cz, float sx, float sy,
                         float sz, const float *angles, int na, int nb, int nv, float SID, float SAD, float da,
                         float ai, float db, float bi, float *sino)
{
    const HostGrid hg = {{nx, ny, nz}, {cx, cy, cz}, {sx, sy, sz}};
    return run(true, vol, hg, angles, na, nb, nv, SID, SAD, da, ai, db, bi, sino);
}

// sino -> vol, accumulated into vol (the reference's atomics; zero it first).
int ref_gpu_backproject_flat(const float *sino, int nx, int ny, int nz, float cx, float cy, float cz, float sx,
                             float sy, float sz, const float *angles, int na, int nb, int nv, float SID, float SAD,
                             float da, float ai, float db, float bi, float *vol)
{
    const HostGrid hg = {{nx, ny, nz}, {cx, cy, cz}, {sx, sy, sz}};
    return run(false, sino, hg, angles, na, nb, nv, SID, SAD, da, ai, db, bi, vol);
}

}  // extern "C"
