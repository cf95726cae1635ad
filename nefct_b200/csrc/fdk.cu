// FDK on sm_100a: cosine + Parker weighting with ramp filtering, and the
// voxel-driven bilinear backprojection with the FDK distance weight.
//
// Filter (mat_codes/filtering.m:5-48, ParkerWeight.m:5-27): the MATLAB code
// zero-pads each detector row to L = max(64, 2^nextpow2(2*nu)), multiplies
// its FFT by the windowed |FFT(ramp)|*2 and crops.  Because the row occupies
// at most L/2 samples the circular convolution never wraps, so it equals the
// direct linear convolution of the row with h = real(IFFT(filter)) over lags
// -(nu-1)..(nu-1).  h is built on the host in FP64 (radix-2 FFT below) with
// the MATLAB scale folded in; the device convolves rows out of shared memory.
//
// Backprojection (nefct/cc/pixel_3d/pixel.cu.cc:12-146 geometry and index
// rules, Q9-Q11, times (src_iso/(src_iso + x'))^2 from
// mat_codes/backprojection.m:12): one thread owns a column of kZ voxels
// along z; per view it computes the column's rotated position, detector
// column and magnification once and then the kZ row taps (one fused
// multiply-add, an exact floor and four gathers per voxel and view).  Views are
// processed in chunks so a chunk's filtered projections stay in L2.
#include <math.h>
#include <algorithm>
#include <complex>
#include <vector>

#include "common.cuh"

namespace nefct {

nefct_status check_cb_geom(const nefct_cb_geom *g);

// ---------------- host: spatial ramp kernel ----------------

static void fft_inplace(std::vector<std::complex<double>> &a, bool inverse)
{
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const double ang = 2.0 * M_PI / (double)len * (inverse ? 1.0 : -1.0);
        const std::complex<double> wl(cos(ang), sin(ang));
        for (size_t i = 0; i < n; i += len) {
            std::complex<double> w(1.0, 0.0);
            for (size_t k = 0; k < len / 2; ++k) {
                const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
                w *= wl;
            }
        }
    }
    if (inverse)
        for (auto &x : a) x /= (double)n;
}

// h_lin[d + na - 1], d = -(na-1)..(na-1): the linear-convolution taps.
static std::vector<float> ramp_taps(int na, int window, double scale)
{
    int p = 0;
    while ((1 << p) < 2 * na) ++p;                      // nextpow2(2*nu)
    const int L = std::max(64, 1 << p);
    // ramp_flat (filtering.m:54-60): nn = -L/2..L/2-1, 1/4 at 0, -1/(pi nn)^2 at odd nn
    std::vector<std::complex<double>> r(L);
    for (int i = 0; i < L; ++i) {
        const int nn = i - L / 2;
        double v = 0.0;
        if (nn == 0) v = 0.25;
        else if (nn & 1) v = -1.0 / ((M_PI * nn) * (M_PI * nn));
        r[i] = v;
    }
    fft_inplace(r, false);
    // Filter (:63-88): 2|FFT|, window on bins 1..L/2, mirror to length L
    std::vector<double> filt(L / 2 + 1);
    for (int k = 0; k <= L / 2; ++k) {
        double f = 2.0 * std::abs(r[k]);
        const double w = 2.0 * M_PI * k / L;
        if (k >= 1) {
            switch (window) {
            case NEFCT_WIN_SHEPP_LOGAN: f *= sin(w / 2.0) / (w / 2.0); break;
            case NEFCT_WIN_COSINE: f *= cos(w / 2.0); break;
            case NEFCT_WIN_HAMMING: f *= 0.54 + 0.46 * cos(w); break;
            case NEFCT_WIN_HANN: f *= (1.0 + cos(w)) / 2.0; break;
            default: break;
            }
        }
        if (w > M_PI) f = 0.0;
        filt[k] = f;
    }
    std::vector<std::complex<double>> full(L);
    for (int k = 0; k <= L / 2; ++k) full[k] = filt[k];
    for (int k = 1; k < L / 2; ++k) full[L - k] = filt[k];
    fft_inplace(full, true);
    std::vector<float> taps(2 * na - 1);
    for (int d = -(na - 1); d <= na - 1; ++d) taps[d + na - 1] = (float)(full[(d + L) % L].real() * scale);
    return taps;
}

// ---------------- device: weighting + row convolution ----------------

static constexpr int kMaxCols = 2048;   // detector columns the filter supports

struct FilterParams {
    int na, nb, nv;
    double src_det;           // DSD
    double da, a_shift, db, b_shift;
    int parker;               // 0 off, +1/-1 = ParkerWeight dir
    double dang;              // view step, degrees
    double fanang;            // ParkerWeight's fanang (half the fan angle), degrees
    float taps[2 * kMaxCols - 1];  // h[d + na - 1], scale folded in (kernel parameter space)
};

static constexpr int kFiltThreads = 128;   // each thread owns 4 consecutive outputs per group
static constexpr int kFiltRows = 4;        // detector rows per CTA (the taps are staged once)

// Shared-memory layout of the filter: taps h[d] for d in [-8, 2na + 8) at
// hs[d + kHPad + off] (zero outside [0, 2na - 2]), off in 0..3 chosen so that
// a thread's tap window starts on a 16-byte boundary; then the weighted row
// x[0..na) with a zero tail to a multiple of 4.
static constexpr int kHPad = 8;
__host__ __device__ static inline int filt_h_floats(int na) { return (2 * na + 2 * kHPad + 4 + 3) & ~3; }
static inline size_t filt_smem_bytes(int na) { return (size_t)(filt_h_floats(na) + ((na + 3) & ~3) + 4) * sizeof(float); }

__global__ void __launch_bounds__(kFiltThreads) fdk_filter_kernel(const __grid_constant__ FilterParams p,
                                                                  const float *__restrict__ sino,
                                                                  float *__restrict__ out)
{
    extern __shared__ __align__(16) float sm[];
    const int na = p.na;
    const int off = (5 - na) & 3;                     // (na - 5 + off) % 4 == 0
    const int hn = filt_h_floats(na);
    float *hs = sm;
    float *x = sm + hn;
    const int na4 = (na + 3) & ~3;
    for (int i = threadIdx.x; i < hn; i += blockDim.x) {
        const int d = i - kHPad - off;
        hs[i] = (d >= 0 && d <= 2 * na - 2) ? p.taps[d] : 0.f;
    }
    const int iv = blockIdx.y;
    for (int row = blockIdx.x * kFiltRows; row < min(p.nb, (blockIdx.x + 1) * kFiltRows); ++row) {
        __syncthreads();                                  // taps staged / previous row consumed
        const double v = ((double)row + p.b_shift) * p.db - (double)p.nb * p.db / 2.0;
        const float *src = sino + ((size_t)iv * p.nb + row) * na;
        for (int j = threadIdx.x; j < na4; j += blockDim.x) {
            if (j >= na) { x[j] = 0.f; continue; }
            const double u = ((double)j + p.a_shift) * p.da - (double)na * p.da / 2.0;
            // cosine weight, filtering.m:10
            double w = p.src_det / sqrt(p.src_det * p.src_det + u * u + v * v);
            if (p.parker) {
                // ParkerWeight.m:5-25 (view i is 1-based there)
                const double as = atan(u / p.src_det) / M_PI * 180.0;
                const double f = p.fanang;
                const double n180 = 180.0 / p.dang;
                const double pw = ((n180 - p.nv) / 2.0 + (iv + 1)) / n180 * 180.0 + p.parker * as;
                if (pw <= f / 2 && pw > -f / 2) {
                    const double s = fmax(sin(M_PI / 2 * (f / 2 + pw) / f), 0.0);
                    w *= s * s;
                }
                if (pw >= 180 - f / 2 && pw < 180 + f / 2) {
                    const double c = fmax(cos(M_PI / 2 * (f / 2 + pw - 180) / f), 0.0);
                    w *= c * c;
                }
                if (pw < -f / 2 || pw > 180 + f / 2) w = 0.0;
            }
            x[j] = (float)((double)src[j] * w);
        }
        __syncthreads();
        float *dst = out + ((size_t)iv * p.nb + row) * na;
        // out[i] = sum_j x[j] h[i - j + na - 1], j ascending for every i.  A
        // thread owns i0..i0+3; per block of four j it needs the taps
        // h[D-3..D+3] (D = i0 + na - 1 - j0), held in an 8-wide register
        // window w[k] = h[D - 4 + k] that slides by four per block (one
        // 16-byte load), with the four x[j] broadcast by one 16-byte load.
        for (int i0 = 4 * threadIdx.x; i0 < na; i0 += 4 * blockDim.x) {
            float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
            const float *hp = hs + kHPad + off + (i0 + na - 5);    // &h[D - 4] for j0 = 0 (16-byte aligned)
            float4 lo = *reinterpret_cast<const float4 *>(hp);     // w0..w3
            float4 hi = *reinterpret_cast<const float4 *>(hp + 4); // w4..w7
            for (int j0 = 0; j0 < na4; j0 += 4) {
                const float4 xv = *reinterpret_cast<const float4 *>(x + j0);
                a0 = fmaf(xv.x, hi.x, a0); a0 = fmaf(xv.y, lo.w, a0); a0 = fmaf(xv.z, lo.z, a0); a0 = fmaf(xv.w, lo.y, a0);
                a1 = fmaf(xv.x, hi.y, a1); a1 = fmaf(xv.y, hi.x, a1); a1 = fmaf(xv.z, lo.w, a1); a1 = fmaf(xv.w, lo.z, a1);
                a2 = fmaf(xv.x, hi.z, a2); a2 = fmaf(xv.y, hi.y, a2); a2 = fmaf(xv.z, hi.x, a2); a2 = fmaf(xv.w, lo.w, a2);
                a3 = fmaf(xv.x, hi.w, a3); a3 = fmaf(xv.y, hi.z, a3); a3 = fmaf(xv.z, hi.y, a3); a3 = fmaf(xv.w, hi.x, a3);
                hp -= 4;
                hi = lo;
                lo = *reinterpret_cast<const float4 *>(hp);
            }
            if (i0 < na) dst[i0] = a0;
            if (i0 + 1 < na) dst[i0 + 1] = a1;
            if (i0 + 2 < na) dst[i0 + 2] = a2;
            if (i0 + 3 < na) dst[i0 + 3] = a3;
        }
    }
}

// ---------------- device: voxel-driven backprojection ----------------

#ifndef NEFCT_FDK_KZ
#define NEFCT_FDK_KZ 4
#endif
static constexpr int kZ = NEFCT_FDK_KZ; // voxels along z per thread
static constexpr int kViewChunk = 32; // views per launch (L2-resident chunk)

struct BpParams {
    int nx, ny, nz, na, nb, nv0, nvc, first;
    float sx, sy, sz, corner_x, corner_y, corner_z;
    float src_iso, src_det, da, ai_p, db, bi_p;
    float inv_da, inv_db, cb;         // 1/da, 1/db and nb/2 - bi_p - 0.5, rounded to float
    int cyl, weight;
    float cs[kViewChunk], sn[kViewChunk];
};

// Per view the column part (rotation, magnification m, detector column a,
// its bilinear weights, the distance weight) follows the reference's
// operations with its divisions replaced by one approximate reciprocal of
// the source distance (a few ulp; every weight is continuous in it);
// (double)(t - ai) - 0.5 rounded to float equals the float subtraction
// t - ai - 0.5f exactly (the double difference is exact), so no FP64 is
// needed.  Per voxel the detector row is b = (m/db) * z + (nb/2 -
// bi - 0.5) by one fused multiply-add (the reference's (m*z)/db + nb/2 - bi
// - 0.5 rounds four times; the two differ by a few ulp of b, which moves the
// bilinear weights continuously), clamped to [-2, nb + 1] (a voxel at the
// source plane has an infinite or NaN b) and floored exactly by the
// magic-constant sum (floor(b) + 1.5*2^23 = round-down(b + 1.5*2^23)).
__global__ void __launch_bounds__(128) fdk_bp_kernel(const __grid_constant__ BpParams p,
                                                     const float *__restrict__ sino, float *__restrict__ vol)
{
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 4 + threadIdx.y;
    const int z0 = blockIdx.z * kZ;
    if (ix >= p.nx || iy >= p.ny) return;
    // voxel centres, pixel.cu.cc:116-118 ((ix + 0.5) * sx / nx + cx, in double)
    const float xc = (float)((ix + 0.5) * (double)p.sx / p.nx + (double)p.corner_x);
    const float yc = (float)((iy + 0.5) * (double)p.sy / p.ny + (double)p.corner_y);
    float zc[kZ], acc[kZ];
    const size_t plane = (size_t)p.nx * p.ny;
    const size_t col = (size_t)iy * p.nx + ix;
#pragma unroll
    for (int k = 0; k < kZ; ++k) {
        const int iz = z0 + k;
        zc[k] = (float)((iz + 0.5) * (double)p.sz / p.nz + (double)p.corner_z);
        acc[k] = (!p.first && iz < p.nz) ? vol[iz * plane + col] : 0.f;
    }
    const float xs = -p.src_iso;
    const float nah = (float)(p.na / 2);   // integer half (Q9)
    const float bhi = (float)(p.nb + 1);
    const unsigned nb1 = (unsigned)(p.nb - 1);
    for (int v = 0; v < p.nvc; ++v) {
        const float cphi = p.cs[v], sphi = p.sn[v];
        const float xc0 = xc * cphi + yc * sphi;
        const float yc0 = -xc * sphi + yc * cphi;
        // 1 / (xc0 - xs) = 1 / (src_iso + xc0): magnification and distance weight share it
        const float inv = rcp_approx(xc0 - xs);
        const float m = p.src_det * inv;                       // SAD / (xc0 - xs)
        float t;
        if (p.cyl) t = atan2f(yc0, xc0 + p.src_iso) * p.inv_da + nah;
        else t = m * yc0 * p.inv_da + nah;
        const float a = __fsub_rn(__fsub_rn(t, p.ai_p), 0.5f);
        const int ia = __float2int_rd(a);
        if (ia < 0 || ia + 1 >= p.na) continue;               // Q11
        const float wa2 = a - (float)ia, wa = 1.f - wa2;
        float u = 1.f;
        if (p.weight) {
            const float r = p.src_iso * inv;
            u = r * r;
        }
        const float bm = m * p.inv_db;
        const float *pv = sino + (size_t)v * p.na * p.nb + ia;
#pragma unroll
        for (int k = 0; k < kZ; ++k) {
            const float b = fminf(fmaxf(fmaf(bm, zc[k], p.cb), -2.f), bhi);
            const float mb = __fadd_rd(b, 12582912.0f);
            const unsigned ib = (unsigned)(__float_as_int(mb) - 0x4B400000);
            if (ib >= nb1) continue;                           // ib < 0 || ib + 1 >= nb
            const float wb2 = b - __fsub_rn(mb, 12582912.0f), wb = 1.f - wb2;
            const float *q = pv + (size_t)ib * p.na;
            const float r0 = fmaf(__ldg(q + 1), wa2, __ldg(q) * wa);
            const float r1 = fmaf(__ldg(q + p.na + 1), wa2, __ldg(q + p.na) * wa);
            acc[k] = fmaf(fmaf(r1, wb2, r0 * wb), u, acc[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < kZ; ++k)
        if (z0 + k < p.nz) vol[(z0 + k) * plane + col] = acc[k];
}

}  // namespace nefct

using namespace nefct;

extern "C" {

nefct_status nefct_fdk_filter(const nefct_cb_geom *g, const float *sino, float *out, int32_t window,
                              int32_t parker, void *stream)
{
    nefct_status st = check_cb_geom(g);
    if (st) return st;
    if (!sino || !out) return fail(NEFCT_ERR_INVALID, "sino and out must be non-NULL");
    if (sino == out) return fail(NEFCT_ERR_INVALID, "fdk filter output may not alias its input");
    if (g->det_kind != NEFCT_DET_FLAT)
        return fail(NEFCT_ERR_UNSUPPORTED, "FDK filtering is defined for flat detectors only (filtering.m)");
    if (window < NEFCT_WIN_RAM_LAK || window > NEFCT_WIN_HANN)
        return fail(NEFCT_ERR_INVALID, "unknown filter window %d", window);
    if (parker < -1 || parker > 1) return fail(NEFCT_ERR_INVALID, "parker must be -1, 0 or 1");
    if (g->na > kMaxCols) return fail(NEFCT_ERR_UNSUPPORTED, "FDK filter supports up to %d detector columns", kMaxCols);
    if (g->src_iso <= 0.f || g->src_det <= 0.f) return fail(NEFCT_ERR_INVALID, "distances must be > 0");
    FilterParams *pp = new FilterParams();
    FilterParams &p = *pp;
    p.na = g->na; p.nb = g->nb; p.nv = g->nv;
    p.src_det = g->src_det;
    p.da = g->da; p.a_shift = g->a_shift; p.db = g->db; p.b_shift = g->b_shift;
    p.parker = parker;
    // scale of filtering.m:43-47: /2/du * dbeta/2 * DSD/DSO
    double dbeta;
    if (parker) {
        if (g->nv < 2) { delete pp; return fail(NEFCT_ERR_INVALID, "Parker weighting needs >= 2 views"); }
        p.dang = fabs((double)g->angles[1] - (double)g->angles[0]) * 180.0 / M_PI;
        if (!(p.dang > 0.0)) { delete pp; return fail(NEFCT_ERR_INVALID, "Parker weighting needs a non-zero view step"); }
        dbeta = 2.0 * M_PI / (180.0 / p.dang);
        const double u0 = (0.0 + g->a_shift) * g->da - g->na * (double)g->da / 2.0;
        const double u1 = (g->na - 1 + (double)g->a_shift) * g->da - g->na * (double)g->da / 2.0;
        p.fanang = fabs(atan(u1 / g->src_det) - atan(u0 / g->src_det)) / M_PI * 180.0 / 2.0;
    } else {
        p.dang = 0.0;
        p.fanang = 0.0;
        dbeta = 2.0 * M_PI / g->nv;
    }
    const double scale = 1.0 / 2.0 / fabs((double)g->da) * dbeta / 2.0 * ((double)g->src_det / g->src_iso);
    std::vector<float> taps = ramp_taps(g->na, window, scale);
    std::copy(taps.begin(), taps.end(), p.taps);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t smem = filt_smem_bytes(g->na);
    fdk_filter_kernel<<<dim3((g->nb + kFiltRows - 1) / kFiltRows, g->nv), kFiltThreads, smem, s>>>(p, sino, out);
    delete pp;
    NEFCT_CHECK_LAUNCH("fdk_filter_kernel");
    return NEFCT_OK;
}

nefct_status nefct_fdk_backproject(const nefct_cb_geom *g, const float *filtered, float *vol, uint32_t flags,
                                   void *stream)
{
    nefct_status st = check_cb_geom(g);
    if (st) return st;
    if (!filtered || !vol) return fail(NEFCT_ERR_INVALID, "filtered and vol must be non-NULL");
    if (flags & ~NEFCT_FDK_NO_WEIGHT) return fail(NEFCT_ERR_INVALID, "unknown flag bits 0x%x", flags);
    BpParams *p = new BpParams();
    p->nx = g->grid.nx; p->ny = g->grid.ny; p->nz = g->grid.nz;
    p->na = g->na; p->nb = g->nb;
    p->sx = g->grid.sx; p->sy = g->grid.sy; p->sz = g->grid.sz;
    // the reference takes the grid's low corner (Q10)
    p->corner_x = g->grid.cx - g->grid.sx / 2.f;
    p->corner_y = g->grid.cy - g->grid.sy / 2.f;
    p->corner_z = g->grid.cz - g->grid.sz / 2.f;
    p->src_iso = g->src_iso; p->src_det = g->src_det;
    // pixel_3d's `ai` is the siddon_3d `ai` minus one half (Q9)
    p->da = g->da; p->ai_p = g->a_shift - 0.5f; p->db = g->db; p->bi_p = g->b_shift - 0.5f;
    p->inv_da = (float)(1.0 / (double)g->da);
    p->inv_db = (float)(1.0 / (double)g->db);
    p->cb = (float)((double)(g->nb / 2) - (double)p->bi_p - 0.5);
    p->cyl = g->det_kind == NEFCT_DET_CYL;
    p->weight = !(flags & NEFCT_FDK_NO_WEIGHT);
    cudaStream_t s = (cudaStream_t)stream;
    dim3 grid((g->grid.nx + 31) / 32, (g->grid.ny + 3) / 4, (g->grid.nz + kZ - 1) / kZ);
    for (int v0 = 0; v0 < g->nv; v0 += kViewChunk) {
        p->nv0 = v0;
        p->nvc = std::min(kViewChunk, g->nv - v0);
        p->first = v0 == 0;
        for (int i = 0; i < p->nvc; ++i) {
            p->cs[i] = (float)cos((double)g->angles[v0 + i]);
            p->sn[i] = (float)sin((double)g->angles[v0 + i]);
        }
        fdk_bp_kernel<<<grid, dim3(32, 4), 0, s>>>(*p, filtered + (size_t)v0 * g->na * g->nb, vol);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { delete p; return cuda_fail(e, "fdk_bp_kernel"); }
    }
    delete p;
    return NEFCT_OK;
}

}  // extern "C"
