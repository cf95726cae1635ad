// TEST INFRASTRUCTURE (oracle/_ref).  Compiles the reference's own CUDA
// device routines and kernels as host C++ so that the oracle restatement
// (nefct_oracle.c) and the GPU kernels can be checked against the
// reference itself.  The reference sources are not copied into this
// repository: oracle/Makefile extracts the line ranges below from the
// reference checkout into oracle/_ref/gen/ at build time (git-ignored).
//
//   siddon3d_fwd.inc  nefct/cc/siddon_3d/siddon.cu.cc:6-390   project_device, Project{Flat,Cyli}Kernel
//   siddon3d_bp.inc   nefct/cc/siddon_3d/siddon.cu.cc:450-832 backproject_device, BackProject{Flat,Cyli}Kernel
//   lor.inc           cpp/siddon/siddon_gpu.cu.cc:6-698       LOR project/backproject + kernels
//   pixel3d.inc       nefct/cc/pixel_3d/pixel.cu.cc:6-146     voxel-driven backprojection
//   deform.inc        cpp/deform/deform.cu.cc:6-46            DeformKernel
//   dd_fdk.inc        nefct/cc/distance_3d/dist_3d_back_fdk.cu.cc:6-255
//                                                             back_project_fdk_kernel (distance-driven)
//
// Kernels run as plain functions: a launch is emulated by setting the
// thread-local blockIdx/threadIdx/blockDim/gridDim and calling the kernel
// once per CUDA thread.  Work is split across OpenMP threads by detector row
// (view, row pairs), so a sample of a few views still keeps every host
// thread busy.  atomicAdd becomes either a plain add on a per-thread private
// volume (private volumes summed in thread order: deterministic for a given
// thread count, used by the tests) or, in the *_atomic entry points, an
// atomic add on the shared output (the host counterpart of the reference's
// device atomics; no per-thread copies of large volumes).
// Build flags: -O3 -fopenmp -ffp-contract=off (no FMA contraction).

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

struct ref_dim3 { unsigned x, y, z; };
static thread_local ref_dim3 blockIdx, threadIdx, blockDim, gridDim;
#define __device__
#define __global__
static thread_local bool tl_shared_atomics = false;
template <class T> static inline T atomicAdd(T *p, T v)
{
    if (tl_shared_atomics) {
        T old, want;
        __atomic_load(p, &old, __ATOMIC_RELAXED);
        do { want = old + v; } while (!__atomic_compare_exchange(p, &old, &want, true, __ATOMIC_RELAXED,
                                                                  __ATOMIC_RELAXED));
        return old;
    }
    T old = *p;
    *p = old + v;
    return old;
}

namespace s3d {
#include "siddon3d_fwd.inc"
#include "siddon3d_bp.inc"
}
#undef abs
namespace lor {
#include "lor.inc"
}
#undef abs
namespace px3 {
#include "pixel3d.inc"
}
#undef abs
namespace dfm {
#include "deform.inc"
}
#undef abs
namespace ddf {
#include "dd_fdk.inc"
}
#undef ABS
#undef MAX
#undef MIN
#undef MAX4
#undef MIN4

// FP64 build of the siddon_3d walk: every float of the included ranges
// becomes double, cosf/sinf become cos/sin.
namespace s3d64 {
#define float double
#define cosf cos
#define sinf sin
#include "siddon3d_fwd.inc"
#include "siddon3d_bp.inc"
#undef float
#undef cosf
#undef sinf
}
#undef abs

static inline void set_thread(unsigned gx, unsigned gy, unsigned gz, unsigned bx, unsigned by,
                              unsigned bz, unsigned i, unsigned j, unsigned k)
{
    blockDim = {bx, by, bz};
    gridDim = {gx, gy, gz};
    blockIdx = {i / bx, j / by, k / bz};
    threadIdx = {i % bx, j % by, k % bz};
}

// Deterministic scatters split their rows into this many chunks, whatever
// the thread count (the restatement uses the same number).
static const int kChunks = 16;

static void sum_private(float *priv, int nth, long long n, float *out)
{
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) {
        float s = 0.0f;
        for (int t = 0; t < nth; ++t) s += priv[(long long)t * n + i];
        out[i] = s;
    }
}

extern "C" {

// project_flat / project_cyli of siddon.cu.cc:392-448 (kernel-level arguments;
// the TF op's da-for-db substitution, Q7, is up to the caller).
void ref_s3d_project(int cyl, const float *image, int nx, int ny, int nz, float cx, float cy, float cz,
                     float sx, float sy, float sz, const float *angles, int na, int nb, int nv,
                     float SID, float SAD, float da, float ai, float db, float bi, float *pv)
{
    const unsigned gx = (na + 15) / 16, gy = (nb + 15) / 16, gz = (nv + 3) / 4;
    memset(pv, 0, sizeof(float) * (size_t)na * nb * nv);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int iv = 0; iv < nv; ++iv)
        for (int ib = 0; ib < nb; ++ib)
            for (int ia = 0; ia < na; ++ia) {
                set_thread(gx, gy, gz, 16, 16, 4, ia, ib, iv);
                if (cyl)
                    s3d::ProjectCyliKernel(image, angles, nx, ny, nz, cx, cy, cz, sx, sy, sz, na, nb, nv,
                                           SID, SAD, da, ai, db, bi, pv);
                else
                    s3d::ProjectFlatKernel(image, angles, nx, ny, nz, cx, cy, cz, sx, sy, sz, na, nb, nv,
                                           SID, SAD, da, ai, db, bi, pv);
            }
}

// One (view, row) of the reference's backprojection kernels: every column ia.
static inline void s3d_bp_row(int cyl, const float *pv, int nx, int ny, int nz, float cx, float cy, float cz,
                              float sx, float sy, float sz, const float *angles, int na, int nb, int nv, float SID,
                              float SAD, float da, float ai, float db, float bi, int iv, int ib, float *dst)
{
    const unsigned gx = (na + 15) / 16, gy = (nb + 15) / 16, gz = (nv + 3) / 4;
    for (int ia = 0; ia < na; ++ia) {
        set_thread(gx, gy, gz, 16, 16, 4, ia, ib, iv);
        // Q8 makes the cylindrical kernel read past the sinogram when nb > nv;
        // the caller passes a buffer padded with zeros for that case.
        if (cyl)
            s3d::BackProjectCyliKernel(pv, angles, nx, ny, nz, cx, cy, cz, sx, sy, sz, na, nb, nv, SID, SAD, da, ai,
                                       db, bi, dst);
        else
            s3d::BackProjectFlatKernel(pv, angles, nx, ny, nz, cx, cy, cz, sx, sy, sz, na, nb, nv, SID, SAD, da, ai,
                                       db, bi, dst);
    }
}

// backproject_flat / backproject_cyli of siddon.cu.cc:834-890 into image
// (overwritten).  The nv*nb (view, row) pairs form kChunks contiguous chunks,
// each scattered in order into its own volume by one thread, and the chunk
// volumes are summed in chunk order: the bits do not depend on the thread
// count, and the restatement's or_cb_backward_f32 splits the same way, so the
// two agree bit for bit.
void ref_s3d_backproject(int cyl, const float *pv, int nx, int ny, int nz, float cx, float cy, float cz,
                         float sx, float sy, float sz, const float *angles, int na, int nb, int nv,
                         float SID, float SAD, float da, float ai, float db, float bi, float *image)
{
    const long long nvox = (long long)nx * ny * nz, rows = (long long)nv * nb;
    float *priv = (float *)calloc((size_t)kChunks * nvox, sizeof(float));
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < kChunks; ++c) {
        tl_shared_atomics = false;
        for (long long r = rows * c / kChunks; r < rows * (c + 1) / kChunks; ++r)
            s3d_bp_row(cyl, pv, nx, ny, nz, cx, cy, cz, sx, sy, sz, angles, na, nb, nv, SID, SAD, da, ai, db, bi,
                       (int)(r / nb), (int)(r % nb), priv + (long long)c * nvox);
    }
    sum_private(priv, kChunks, nvox, image);
    free(priv);
}

// The same backprojection with atomic adds into the shared, zeroed image
// (the host form of the reference's device atomicAdd): no private volumes,
// (view, row) pairs handed out dynamically.  The summation order depends on
// scheduling, as on the GPU.
void ref_s3d_backproject_atomic(int cyl, const float *pv, int nx, int ny, int nz, float cx, float cy, float cz,
                                float sx, float sy, float sz, const float *angles, int na, int nb, int nv,
                                float SID, float SAD, float da, float ai, float db, float bi, float *image)
{
    const long long nvox = (long long)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nvox; ++i) image[i] = 0.0f;
#pragma omp parallel
    {
        tl_shared_atomics = true;
#pragma omp for collapse(2) schedule(dynamic, 1)
        for (int iv = 0; iv < nv; ++iv)
            for (int ib = 0; ib < nb; ++ib)
                s3d_bp_row(cyl, pv, nx, ny, nz, cx, cy, cz, sx, sy, sz, angles, na, nb, nv, SID, SAD, da, ai, db,
                           bi, iv, ib, image);
        tl_shared_atomics = false;
    }
}

// Threads the OpenMP runtime of this library uses.
int ref_max_threads(void) { return omp_get_max_threads(); }

// FP64 builds of the same two entry points.
void ref_s3d_project_f64(int cyl, const double *image, int nx, int ny, int nz, double cx, double cy,
                         double cz, double sx, double sy, double sz, const double *angles, int na, int nb,
                         int nv, double SID, double SAD, double da, double ai, double db, double bi,
                         double *pv)
{
    const unsigned gx = (na + 15) / 16, gy = (nb + 15) / 16, gz = (nv + 3) / 4;
    memset(pv, 0, sizeof(double) * (size_t)na * nb * nv);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int iv = 0; iv < nv; ++iv)
        for (int ib = 0; ib < nb; ++ib)
            for (int ia = 0; ia < na; ++ia) {
                set_thread(gx, gy, gz, 16, 16, 4, ia, ib, iv);
                if (cyl)
                    s3d64::ProjectCyliKernel(image, angles, nx, ny, nz, cx, cy, cz, sx, sy, sz, na, nb, nv,
                                             SID, SAD, da, ai, db, bi, pv);
                else
                    s3d64::ProjectFlatKernel(image, angles, nx, ny, nz, cx, cy, cz, sx, sy, sz, na, nb, nv,
                                             SID, SAD, da, ai, db, bi, pv);
            }
}

void ref_s3d_backproject_f64(int cyl, const double *pv, int nx, int ny, int nz, double cx, double cy,
                             double cz, double sx, double sy, double sz, const double *angles, int na,
                             int nb, int nv, double SID, double SAD, double da, double ai, double db,
                             double bi, double *image)
{
    const unsigned gx = (na + 15) / 16, gy = (nb + 15) / 16, gz = (nv + 3) / 4;
    const long long nvox = (long long)nx * ny * nz;
    memset(image, 0, sizeof(double) * (size_t)nvox);
    for (int iv = 0; iv < nv; ++iv)
        for (int ib = 0; ib < nb; ++ib)
            for (int ia = 0; ia < na; ++ia) {
                set_thread(gx, gy, gz, 16, 16, 4, ia, ib, iv);
                if (cyl)
                    s3d64::BackProjectCyliKernel(pv, angles, nx, ny, nz, cx, cy, cz, sx, sy, sz, na, nb, nv,
                                                 SID, SAD, da, ai, db, bi, image);
                else
                    s3d64::BackProjectFlatKernel(pv, angles, nx, ny, nz, cx, cy, cz, sx, sy, sz, na, nb, nv,
                                                 SID, SAD, da, ai, db, bi, image);
            }
}

// projection() of cpp/siddon/siddon_gpu.cu.cc:700-722; lors is [6][n].
// Rays that the reference leaves unwritten (Q4) keep the caller's values.
void ref_lor_project(const float *lors, long long n, const float *image, int nx, int ny, int nz,
                     float cx, float cy, float cz, float sx, float sy, float sz, float *vproj)
{
    const unsigned G = 32, B = 1024;
#pragma omp parallel for schedule(static)
    for (long long t = 0; t < (long long)G * B; ++t) {
        set_thread(G, 1, 1, B, 1, 1, (unsigned)t, 0, 0);
        lor::ProjectKernel(lors, lors + n, lors + 2 * n, lors + 3 * n, lors + 4 * n, lors + 5 * n,
                           nx, ny, nz, cx, cy, cz, sx, sy, sz, (int)n, image, vproj);
    }
}

// backprojection() of siddon_gpu.cu.cc:725-747 into image (overwritten; the
// reference op accumulates into an unzeroed buffer, Q6).
void ref_lor_backproject(const float *lors, long long n, const float *vproj, int nx, int ny, int nz,
                         float cx, float cy, float cz, float sx, float sy, float sz, float *image)
{
    const unsigned G = 32, B = 1024;
    const long long nvox = (long long)nx * ny * nz, T = (long long)G * B;
    float *priv = (float *)calloc((size_t)kChunks * nvox, sizeof(float));
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < kChunks; ++c) {
        for (long long t = T * c / kChunks; t < T * (c + 1) / kChunks; ++t) {
            set_thread(G, 1, 1, B, 1, 1, (unsigned)t, 0, 0);
            lor::BackProjectKernel(lors, lors + n, lors + 2 * n, lors + 3 * n, lors + 4 * n, lors + 5 * n,
                                   nx, ny, nz, cx, cy, cz, sx, sy, sz, (int)n, vproj, priv + (long long)c * nvox);
        }
    }
    sum_private(priv, kChunks, nvox, image);
    free(priv);
}

// backproject_flat / backproject_cyli of pixel.cu.cc:148-204; `corner` is the
// reference's `center` argument (the grid's low corner, Q10).
void ref_pixel_backproject(int cyl, const float *pv, int nx, int ny, int nz, const float *corner,
                           const float *size, const float *angles, int na, int nb, int nv, float SID,
                           float SAD, float da, float ai, float db, float bi, float *image)
{
    const unsigned gx = (nx + 15) / 16, gy = (ny + 15) / 16, gz = (nz + 3) / 4;
    memset(image, 0, sizeof(float) * (size_t)nx * ny * nz);
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                set_thread(gx, gy, gz, 16, 16, 4, ix, iy, iz);
                if (cyl)
                    px3::BackProjectCyliKernel(pv, angles, nx, ny, nz, corner[0], corner[1], corner[2],
                                               size[0], size[1], size[2], na, nb, nv, SID, SAD, da, ai,
                                               db, bi, image);
                else
                    px3::BackProjectFlatKernel(pv, angles, nx, ny, nz, corner[0], corner[1], corner[2],
                                               size[0], size[1], size[2], na, nb, nv, SID, SAD, da, ai,
                                               db, bi, image);
            }
}

// deform() of cpp/deform/deform.cu.cc:112-126.  The reference op does not
// clear its output (Q13); img1 is cleared here first.
void ref_deform(const float *img, const float *mx, const float *my, const float *mz, int nx, int ny,
                int nz, float *img1)
{
    const unsigned gx = (nx + 15) / 16, gy = (ny + 15) / 16, gz = (nz + 3) / 4;
    memset(img1, 0, sizeof(float) * (size_t)nx * ny * nz);
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                set_thread(gx, gy, gz, 16, 16, 4, ix, iy, iz);
                dfm::DeformKernel(img, mx, my, mz, nx, ny, nz, img1);
            }
}

// back_project_flat_fdk_gpu / back_project_cyli_fdk_gpu of
// dist_3d_back_fdk.cu.cc:257-298 into image (overwritten; the reference
// accumulates into the caller's buffer).  (view, row) pairs in kChunks
// fixed chunks summed in chunk order, like the restatement's
// or_dd_backproject_f32.  SID = source-detector, SAD =
// source-axis (python naming there); voxel units, grid centred on the axis.
void ref_dd_backproject(int cyl, const float *pv, int nx, int ny, int nz, const float *offsets,
                        const float *angles, int nv, float SID, float SAD, float da, float ai, int na, float db,
                        float bi, int nb, float *image)
{
    const unsigned gx = (na + 15) / 16, gy = (nb + 15) / 16, gz = (nv + 3) / 4;
    const long long nvox = (long long)nx * ny * nz, rows = (long long)nv * nb;
    float *priv = (float *)calloc((size_t)kChunks * nvox, sizeof(float));
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < kChunks; ++c) {
        float *mine = priv + (long long)c * nvox;
        for (long long r = rows * c / kChunks; r < rows * (c + 1) / kChunks; ++r) {
            const int iv = (int)(r / nb), ib = (int)(r % nb);
            for (int ia = 0; ia < na; ++ia) {
                set_thread(gx, gy, gz, 16, 16, 4, ia, ib, iv);
                ddf::back_project_fdk_kernel(cyl, angles, offsets, nv, SID, SAD, nx, ny, nz, da, ai, na, db, bi, nb,
                                             pv, mine);
            }
        }
    }
    sum_private(priv, kChunks, nvox, image);
    free(priv);
}

}  // extern "C"
