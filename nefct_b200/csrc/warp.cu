// Trilinear deformation warp of cpp/deform on sm_100a, with the two
// derivatives the differentiable 4D path needs.
//
// Forward (DeformKernel, cpp/deform/deform.cu.cc:13-46): voxel i samples img
// at i + m[i] (voxel units).  The reference rejects a sample when its base
// index is <= 0 or its upper tap is out of range (Q13) and then leaves the
// output unwritten; here such voxels are written as 0.  The eight taps are
// summed in the reference's order.
//
// Adjoint with respect to img: every in-range sample scatters its eight
// weighted taps (atomics; each voxel's taps are a 2x2x2 neighbourhood, so
// neighbouring threads hit neighbouring addresses).  Gradient with respect to
// m: the analytic derivative of the trilinear weights, gathered.  Threads run
// x-fastest so the field reads are coalesced.
#include "common.cuh"

namespace nefct {

template <typename T> struct Tap {
    int base;                 // flat index of the (xi, yi, zi) corner
    T fx, fy, fz;             // fractional offsets (wx2, wy2, wz2)
    bool ok;
};

template <typename T>
__device__ __forceinline__ Tap<T> warp_tap(int ix, int iy, int iz, T mx, T my, T mz, int nx, int ny, int nz)
{
    Tap<T> t;
    const T px = (T)ix + mx, py = (T)iy + my, pz = (T)iz + mz;
    const int xi = FP<T>::ifloor(px), yi = FP<T>::ifloor(py), zi = FP<T>::ifloor(pz);
    // Q13: deform.cu.cc:31-33
    t.ok = !(xi <= 0 || xi + 1 >= nx || yi <= 0 || yi + 1 >= ny || zi <= 0 || zi + 1 >= nz);
    t.fx = px - (T)xi; t.fy = py - (T)yi; t.fz = pz - (T)zi;
    t.base = t.ok ? xi + yi * nx + zi * nx * ny : 0;
    return t;
}

#ifndef NEFCT_WARP_VPT
#define NEFCT_WARP_VPT 2
#endif
// Voxels per thread of the forward (x-strided by 32, so every load stays
// coalesced): a thread issues the field reads of all its voxels, then all
// their tap gathers, before it sums any -- more loads in flight per thread.
// Measured (fields and image larger than L2): 1 / 2 / 4 / 8 voxels per
// thread take 0.78 / 0.70 / 0.96 / 1.62 ms at 512^3 (25 / 32 / 64 / 128
// registers).
static constexpr int kWarpVpt = NEFCT_WARP_VPT;

template <typename T, int VPT>
__global__ void __launch_bounds__(256) warp_forward_kernel(const T *__restrict__ img, const T *__restrict__ mx,
                                                           const T *__restrict__ my, const T *__restrict__ mz,
                                                           int nx, int ny, int nz, T *__restrict__ out)
{
    const int x0 = blockIdx.x * (32 * VPT) + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y, iz = blockIdx.z;
    if (iy >= ny) return;
    const int row = iy * nx + iz * nx * ny;
    const int sy = nx, sz = nx * ny;
    Tap<T> t[VPT];
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
        const int ix = x0 + 32 * k;
        t[k] = ix < nx ? warp_tap<T>(ix, iy, iz, mx[row + ix], my[row + ix], mz[row + ix], nx, ny, nz) : Tap<T>{0};
    }
    T c[VPT][8];
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
        const T *b = img + t[k].base;
        const bool ok = t[k].ok;
        c[k][0] = ok ? __ldg(b) : (T)0;
        c[k][1] = ok ? __ldg(b + sz) : (T)0;
        c[k][2] = ok ? __ldg(b + sy) : (T)0;
        c[k][3] = ok ? __ldg(b + sy + sz) : (T)0;
        c[k][4] = ok ? __ldg(b + 1) : (T)0;
        c[k][5] = ok ? __ldg(b + 1 + sz) : (T)0;
        c[k][6] = ok ? __ldg(b + 1 + sy) : (T)0;
        c[k][7] = ok ? __ldg(b + 1 + sy + sz) : (T)0;
    }
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
        const int ix = x0 + 32 * k;
        if (ix >= nx) continue;
        T v = (T)0;
        if (t[k].ok) {
            const T wx2 = t[k].fx, wx = (T)1 - wx2, wy2 = t[k].fy, wy = (T)1 - wy2, wz2 = t[k].fz, wz = (T)1 - wz2;
            v = c[k][0] * wx * wy * wz + c[k][1] * wx * wy * wz2 + c[k][2] * wx * wy2 * wz +
                c[k][3] * wx * wy2 * wz2 + c[k][4] * wx2 * wy * wz +
                c[k][5] * wx2 * wy * wz2 + c[k][6] * wx2 * wy2 * wz +
                c[k][7] * wx2 * wy2 * wz2;
        }
        out[row + ix] = v;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) warp_adjoint_kernel(const T *__restrict__ gout, const T *__restrict__ mx,
                                                           const T *__restrict__ my, const T *__restrict__ mz,
                                                           int nx, int ny, int nz, T *__restrict__ gimg)
{
    const int ix = blockIdx.x * 32 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y, iz = blockIdx.z;
    if (ix >= nx || iy >= ny) return;
    const int id = ix + iy * nx + iz * nx * ny;
    const T g = gout[id];
    if (g == (T)0) return;
    const Tap<T> t = warp_tap<T>(ix, iy, iz, mx[id], my[id], mz[id], nx, ny, nz);
    if (!t.ok) return;
    const int sy = nx, sz = nx * ny;
    const T wx2 = t.fx, wx = (T)1 - wx2, wy2 = t.fy, wy = (T)1 - wy2, wz2 = t.fz, wz = (T)1 - wz2;
    T *b = gimg + t.base;
    atomicAdd(b, g * (wx * wy * wz));
    atomicAdd(b + sz, g * (wx * wy * wz2));
    atomicAdd(b + sy, g * (wx * wy2 * wz));
    atomicAdd(b + sy + sz, g * (wx * wy2 * wz2));
    atomicAdd(b + 1, g * (wx2 * wy * wz));
    atomicAdd(b + 1 + sz, g * (wx2 * wy * wz2));
    atomicAdd(b + 1 + sy, g * (wx2 * wy2 * wz));
    atomicAdd(b + 1 + sy + sz, g * (wx2 * wy2 * wz2));
}

template <typename T>
__global__ void __launch_bounds__(256) warp_grad_dvf_kernel(const T *__restrict__ img, const T *__restrict__ mx,
                                                            const T *__restrict__ my, const T *__restrict__ mz,
                                                            const T *__restrict__ gout, int nx, int ny, int nz,
                                                            T *__restrict__ gmx, T *__restrict__ gmy,
                                                            T *__restrict__ gmz)
{
    const int ix = blockIdx.x * 32 + threadIdx.x, iy = blockIdx.y * 8 + threadIdx.y, iz = blockIdx.z;
    if (ix >= nx || iy >= ny) return;
    const int id = ix + iy * nx + iz * nx * ny;
    const Tap<T> t = warp_tap<T>(ix, iy, iz, mx[id], my[id], mz[id], nx, ny, nz);
    T gx = (T)0, gy = (T)0, gz = (T)0;
    const T g = gout[id];
    if (t.ok && g != (T)0) {
        const int sy = nx, sz = nx * ny;
        const T *b = img + t.base;
        const T c000 = __ldg(b), c001 = __ldg(b + sz), c010 = __ldg(b + sy), c011 = __ldg(b + sy + sz);
        const T c100 = __ldg(b + 1), c101 = __ldg(b + 1 + sz), c110 = __ldg(b + 1 + sy),
                c111 = __ldg(b + 1 + sy + sz);   // c[x][y][z]
        const T fx = t.fx, fy = t.fy, fz = t.fz;
        const T ux = (T)1 - fx, uy = (T)1 - fy, uz = (T)1 - fz;
        // d/dfx of sum c * wx * wy * wz with wx = 1 - fx, wx2 = fx
        const T ex0 = (c000 * uy + c010 * fy) * uz + (c001 * uy + c011 * fy) * fz;
        const T ex1 = (c100 * uy + c110 * fy) * uz + (c101 * uy + c111 * fy) * fz;
        gx = g * (ex1 - ex0);
        const T ey0 = (c000 * ux + c100 * fx) * uz + (c001 * ux + c101 * fx) * fz;
        const T ey1 = (c010 * ux + c110 * fx) * uz + (c011 * ux + c111 * fx) * fz;
        gy = g * (ey1 - ey0);
        const T ez0 = (c000 * ux + c100 * fx) * uy + (c010 * ux + c110 * fx) * fy;
        const T ez1 = (c001 * ux + c101 * fx) * uy + (c011 * ux + c111 * fx) * fy;
        gz = g * (ez1 - ez0);
    }
    gmx[id] = gx;
    gmy[id] = gy;
    gmz[id] = gz;
}


// Displacement-field inversion of nefct/cc/deform/deform_tex.cu.cc:78-99:
// starting from 0, `iters` Gauss-Seidel fixed-point passes
//   x <- -mx(p + (x, y, z)),  y <- -my(...),  z <- -mz(...)
// sampled trilinearly with clamp-to-edge addressing (the reference samples a
// linear-filtered, clamp-addressed texture at texel centres; hardware
// filtering keeps 8 fractional bits of the weights, this samples in FP32).
__device__ __forceinline__ float clamp_lerp3(const float *__restrict__ m, float px, float py, float pz, int nx, int ny,
                                             int nz)
{
    const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
    const float ax = px - fx, ay = py - fy, az = pz - fz;
    const int x0 = min(max((int)fx, 0), nx - 1), x1 = min(max((int)fx + 1, 0), nx - 1);
    const int y0 = min(max((int)fy, 0), ny - 1), y1 = min(max((int)fy + 1, 0), ny - 1);
    const int z0 = min(max((int)fz, 0), nz - 1), z1 = min(max((int)fz + 1, 0), nz - 1);
    const size_t sy = nx, sz = (size_t)nx * ny;
    const float c00 = __ldg(m + x0 + y0 * sy + z0 * sz) * (1.f - ax) + __ldg(m + x1 + y0 * sy + z0 * sz) * ax;
    const float c10 = __ldg(m + x0 + y1 * sy + z0 * sz) * (1.f - ax) + __ldg(m + x1 + y1 * sy + z0 * sz) * ax;
    const float c01 = __ldg(m + x0 + y0 * sy + z1 * sz) * (1.f - ax) + __ldg(m + x1 + y0 * sy + z1 * sz) * ax;
    const float c11 = __ldg(m + x0 + y1 * sy + z1 * sz) * (1.f - ax) + __ldg(m + x1 + y1 * sy + z1 * sz) * ax;
    const float c0 = c00 * (1.f - ay) + c10 * ay, c1 = c01 * (1.f - ay) + c11 * ay;
    return c0 * (1.f - az) + c1 * az;
}

__global__ void __launch_bounds__(256) warp_invert_kernel(const float *__restrict__ mx, const float *__restrict__ my,
                                                          const float *__restrict__ mz, int nx, int ny, int nz,
                                                          int iters, float *ix, float *iy, float *iz)
{
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x >= nx || y >= ny) return;
    float u = 0.f, v = 0.f, w = 0.f;
    for (int it = 0; it < iters; ++it) {
        u = -clamp_lerp3(mx, x + u, y + v, z + w, nx, ny, nz);
        v = -clamp_lerp3(my, x + u, y + v, z + w, nx, ny, nz);
        w = -clamp_lerp3(mz, x + u, y + v, z + w, nx, ny, nz);
    }
    const size_t id = x + (size_t)y * nx + (size_t)z * nx * ny;
    ix[id] = u;
    iy[id] = v;
    iz[id] = w;
}

static nefct_status check_warp(int nx, int ny, int nz)
{
    if (nx < 1 || ny < 1 || nz < 1) return fail(NEFCT_ERR_INVALID, "warp grid must be >= 1 (got %d x %d x %d)", nx, ny, nz);
    if ((long long)nx * ny * nz >= (1ll << 31)) return fail(NEFCT_ERR_INVALID, "warp grid too large");
    if (nz > 65535) return fail(NEFCT_ERR_INVALID, "nz must be <= 65535");
    return NEFCT_OK;
}

template <typename T>
static nefct_status warp_forward_impl(const T *img, const T *mx, const T *my, const T *mz, int nx, int ny, int nz,
                                      T *out, cudaStream_t s)
{
    nefct_status st = check_warp(nx, ny, nz);
    if (st) return st;
    if (!img || !mx || !my || !mz || !out) return fail(NEFCT_ERR_INVALID, "NULL buffer");
    warp_forward_kernel<T, kWarpVpt><<<dim3((nx + 32 * kWarpVpt - 1) / (32 * kWarpVpt), (ny + 7) / 8, nz), dim3(32, 8), 0, s>>>(
        img, mx, my, mz, nx, ny, nz, out);
    NEFCT_CHECK_LAUNCH("warp_forward_kernel");
    return NEFCT_OK;
}

template <typename T>
static nefct_status warp_adjoint_impl(const T *gout, const T *mx, const T *my, const T *mz, int nx, int ny, int nz,
                                      T *gimg, cudaStream_t s)
{
    nefct_status st = check_warp(nx, ny, nz);
    if (st) return st;
    if (!gout || !mx || !my || !mz || !gimg) return fail(NEFCT_ERR_INVALID, "NULL buffer");
    NEFCT_CHECK_CUDA(cudaMemsetAsync(gimg, 0, (size_t)nx * ny * nz * sizeof(T), s));
    warp_adjoint_kernel<T><<<dim3((nx + 31) / 32, (ny + 7) / 8, nz), dim3(32, 8), 0, s>>>(gout, mx, my, mz, nx, ny, nz, gimg);
    NEFCT_CHECK_LAUNCH("warp_adjoint_kernel");
    return NEFCT_OK;
}

template <typename T>
static nefct_status warp_grad_impl(const T *img, const T *mx, const T *my, const T *mz, const T *gout, int nx,
                                   int ny, int nz, T *gmx, T *gmy, T *gmz, cudaStream_t s)
{
    nefct_status st = check_warp(nx, ny, nz);
    if (st) return st;
    if (!img || !mx || !my || !mz || !gout || !gmx || !gmy || !gmz) return fail(NEFCT_ERR_INVALID, "NULL buffer");
    warp_grad_dvf_kernel<T><<<dim3((nx + 31) / 32, (ny + 7) / 8, nz), dim3(32, 8), 0, s>>>(
        img, mx, my, mz, gout, nx, ny, nz, gmx, gmy, gmz);
    NEFCT_CHECK_LAUNCH("warp_grad_dvf_kernel");
    return NEFCT_OK;
}

}  // namespace nefct

using namespace nefct;

extern "C" {

nefct_status nefct_warp_forward(const float *img, const float *mx, const float *my, const float *mz, int32_t nx,
                                int32_t ny, int32_t nz, float *out, void *stream)
{
    return warp_forward_impl<float>(img, mx, my, mz, nx, ny, nz, out, (cudaStream_t)stream);
}

nefct_status nefct_warp_adjoint(const float *gout, const float *mx, const float *my, const float *mz, int32_t nx,
                                int32_t ny, int32_t nz, float *gimg, void *stream)
{
    return warp_adjoint_impl<float>(gout, mx, my, mz, nx, ny, nz, gimg, (cudaStream_t)stream);
}

nefct_status nefct_warp_grad_dvf(const float *img, const float *mx, const float *my, const float *mz,
                                 const float *gout, int32_t nx, int32_t ny, int32_t nz, float *gmx, float *gmy,
                                 float *gmz, void *stream)
{
    return warp_grad_impl<float>(img, mx, my, mz, gout, nx, ny, nz, gmx, gmy, gmz, (cudaStream_t)stream);
}

nefct_status nefct_warp_forward_f64(const double *img, const double *mx, const double *my, const double *mz,
                                    int32_t nx, int32_t ny, int32_t nz, double *out, void *stream)
{
    return warp_forward_impl<double>(img, mx, my, mz, nx, ny, nz, out, (cudaStream_t)stream);
}

nefct_status nefct_warp_adjoint_f64(const double *gout, const double *mx, const double *my, const double *mz,
                                    int32_t nx, int32_t ny, int32_t nz, double *gimg, void *stream)
{
    return warp_adjoint_impl<double>(gout, mx, my, mz, nx, ny, nz, gimg, (cudaStream_t)stream);
}

nefct_status nefct_warp_grad_dvf_f64(const double *img, const double *mx, const double *my, const double *mz,
                                     const double *gout, int32_t nx, int32_t ny, int32_t nz, double *gmx,
                                     double *gmy, double *gmz, void *stream)
{
    return warp_grad_impl<double>(img, mx, my, mz, gout, nx, ny, nz, gmx, gmy, gmz, (cudaStream_t)stream);
}

nefct_status nefct_warp_invert(const float *mx, const float *my, const float *mz, int32_t nx, int32_t ny, int32_t nz,
                               int32_t iters, float *ix, float *iy, float *iz, void *stream)
{
    nefct_status st = check_warp(nx, ny, nz);
    if (st) return st;
    if (!mx || !my || !mz || !ix || !iy || !iz) return fail(NEFCT_ERR_INVALID, "NULL buffer");
    if (iters < 0 || iters > 10000) return fail(NEFCT_ERR_INVALID, "iters must be in [0, 10000]");
    warp_invert_kernel<<<dim3((nx + 31) / 32, (ny + 7) / 8, nz), dim3(32, 8), 0, (cudaStream_t)stream>>>(
        mx, my, mz, nx, ny, nz, iters, ix, iy, iz);
    NEFCT_CHECK_LAUNCH("warp_invert_kernel");
    return NEFCT_OK;
}

}  // extern "C"
