// TEST INFRASTRUCTURE: the reference's own CUDA kernels and their host
// launchers, built unchanged by nvcc from the reference checkout (the
// Makefile extracts the line ranges into _ref/gen/):
//   siddon3d_gpu.inc  nefct/cc/siddon_3d/siddon.cu.cc:6-890 (cone-beam pair)
//   pixel3d_gpu.inc   nefct/cc/pixel_3d/pixel.cu.cc:6-204 (voxel-driven
//                     backprojection)
//   lor_gpu.inc       cpp/siddon/siddon_gpu.cu.cc:6-747 (LOR pair)
//   dd_fdk_gpu.inc    nefct/cc/distance_3d/dist_3d_back_fdk.cu.cc:6-298
//                     (distance-driven FDK backprojection)
//   deform_gpu.inc    cpp/deform/deform.cu.cc:6-126 (trilinear warp)
// Each file sits in its own namespace (they share function names).  It runs
// the reference's own CUDA path on the GPU for the parity tests and for
// timing that path beside the library's.  Only tests load it.
//
// Read before running: every volume access and atomicAdd of these kernels
// sits behind range checks of its indices (0 <= c < n, with the neighbour
// index checked on its open side); pixel_3d reads its four taps only when
// ia >= 0, ia + 1 < na, ib >= 0, ib + 1 < nb; the flat sinogram index
// ia + ib*na + iv*na*nb and the LOR index tid < num_events stay in their
// buffers.  The cylindrical siddon_3d backprojection reads its sinogram at
// ia + iv*na + ib*na*nb (quirk Q8, siddon.cu.cc:830), which leaves the
// buffer when nb > nv, so only the flat variants are exported.  The
// distance-driven kernel adds into voxels ix < nx, max(0, Yi1) <= iy <=
// min(ny - 1, Yi2), max(0, Zi1) <= iz <= min(nz - 1, Zi2) and reads its bin
// id < na*nb*nv; the warp reads its 8 taps only when 0 < xi, xi + 1 < nx
// (and the same in y, z).
#include <cuda_runtime.h>
#include <stddef.h>

namespace s3d {
#include "siddon3d_gpu.inc"
}
#undef abs
namespace px3 {
#include "pixel3d_gpu.inc"
}
#undef abs
namespace lor {
#include "lor_gpu.inc"
}
#undef abs
namespace ddf {
#include "dd_fdk_gpu.inc"
}
#undef ABS
#undef MAX
#undef MIN
#undef MAX4
#undef MIN4
namespace dfm {
#include "deform_gpu.inc"
}
#undef abs

namespace {

struct HostGrid {
    int dims[3];
    float center[3];
    float size[3];
};

// The reference's host functions read grid / center / size back from the
// device (e.g. siddon.cu.cc:401-406), so they are staged in one device block.
// Everything runs on the legacy default stream like the reference; the
// call synchronises and returns the CUDA error code (0 = success).
template <class Fn> int with_grid(const HostGrid &hg, Fn fn)
{
    unsigned char *blk = nullptr;
    cudaError_t e = cudaMalloc(&blk, sizeof(HostGrid));
    if (e != cudaSuccess) return (int)e;
    e = cudaMemcpy(blk, &hg, sizeof(HostGrid), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        fn((const int *)blk, (const float *)(blk + offsetof(HostGrid, center)),
           (const float *)(blk + offsetof(HostGrid, size)));
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    cudaFree(blk);
    return (int)e;
}

}  // namespace

extern "C" {

// siddon_3d flat pair.  vol: device [nz][ny][nx]; angles: device [nv];
// sino: device [nv][nb][na].  Kernel naming (SID source-isocentre, SAD
// source-detector), grid given by its centre.  The backprojection
// accumulates into vol (the reference's atomics; zero it first).
int ref_gpu_project_flat(const float *vol, int nx, int ny, int nz, float cx, float cy, float cz, float sx, float sy,
                         float sz, const float *angles, int na, int nb, int nv, float SID, float SAD, float da,
                         float ai, float db, float bi, float *sino)
{
    return with_grid({{nx, ny, nz}, {cx, cy, cz}, {sx, sy, sz}}, [&](const int *g, const float *c, const float *s) {
        s3d::project_flat(vol, g, c, s, angles, na, nb, nv, SID, SAD, da, ai, db, bi, sino);
    });
}

int ref_gpu_backproject_flat(const float *sino, int nx, int ny, int nz, float cx, float cy, float cz, float sx,
                             float sy, float sz, const float *angles, int na, int nb, int nv, float SID, float SAD,
                             float da, float ai, float db, float bi, float *vol)
{
    return with_grid({{nx, ny, nz}, {cx, cy, cz}, {sx, sy, sz}}, [&](const int *g, const float *c, const float *s) {
        s3d::backproject_flat(sino, g, c, s, angles, na, nb, nv, SID, SAD, da, ai, db, bi, vol);
    });
}

// pixel_3d flat backprojection (pixel.cu.cc:148-175): the grid is given by
// its low corner (quirk Q10); accumulates into vol (zero it first).
int ref_gpu_pixel_backproject_flat(const float *sino, int nx, int ny, int nz, float x0, float y0, float z0, float sx,
                                   float sy, float sz, const float *angles, int na, int nb, int nv, float SID,
                                   float SAD, float da, float ai, float db, float bi, float *vol)
{
    return with_grid({{nx, ny, nz}, {x0, y0, z0}, {sx, sy, sz}}, [&](const int *g, const float *c, const float *s) {
        px3::backproject_flat(sino, g, c, s, angles, na, nb, nv, SID, SAD, da, ai, db, bi, vol);
    });
}

// cpp/siddon LOR pair (siddon_gpu.cu.cc:700-747).  lors: device [6][n] rows
// x1 y1 z1 x2 y2 z2.  The forward writes out[i] except for the lines it
// skips (quirk Q4: zero out first); the backprojection accumulates into vol
// (quirk Q6: zero it first).
int ref_gpu_lor_forward(const float *lors, int n, int nx, int ny, int nz, float cx, float cy, float cz, float sx,
                        float sy, float sz, const float *vol, float *out)
{
    const size_t r = (size_t)n;
    return with_grid({{nx, ny, nz}, {cx, cy, cz}, {sx, sy, sz}}, [&](const int *g, const float *c, const float *s) {
        lor::projection(lors, lors + r, lors + 2 * r, lors + 3 * r, lors + 4 * r, lors + 5 * r, out, g, c, s, vol, n);
    });
}

int ref_gpu_lor_backward(const float *lors, int n, int nx, int ny, int nz, float cx, float cy, float cz, float sx,
                         float sy, float sz, const float *vals, float *vol)
{
    const size_t r = (size_t)n;
    return with_grid({{nx, ny, nz}, {cx, cy, cz}, {sx, sy, sz}}, [&](const int *g, const float *c, const float *s) {
        lor::backprojection(lors, lors + r, lors + 2 * r, lors + 3 * r, lors + 4 * r, lors + 5 * r, vals, g, c, s, vol,
                            n);
    });
}

// dist_3d_back_fdk.cu.cc:257-276 (flat detector), the reference's naming
// (SID source-detector, SAD source-axis, voxel units): proj device
// [nv][nb][na], offsets / angles device [nv]; adds into vol [nz][ny][nx]
// (zero it first).
int ref_gpu_dd_backproject_flat(const float *proj, int nx, int ny, int nz, const float *offsets, const float *angles,
                                int nv, float SID, float SAD, float da, float ai, int na, float db, float bi, int nb,
                                float *vol)
{
    const HostGrid hg = {{nx, ny, nz}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    return with_grid(hg, [&](const int *g, const float *, const float *) {
        ddf::back_project_flat_fdk_gpu(proj, g, offsets, angles, nv, SID, SAD, da, ai, na, db, bi, nb, vol);
    });
}

// cpp/deform deform (deform.cu.cc:112-126): img, mx, my, mz, out device
// [nz][ny][nx]; out is written where the reference writes (Q13: zero it
// first).
int ref_gpu_deform(const float *img, const float *mx, const float *my, const float *mz, int nx, int ny, int nz,
                   float *out)
{
    const HostGrid hg = {{nx, ny, nz}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    return with_grid(hg, [&](const int *g, const float *, const float *) { dfm::deform(img, mx, my, mz, g, out); });
}

}  // extern "C"
