// FDK on sm_100a: cosine + Parker weighting with ramp filtering, and the
// voxel-driven bilinear backprojection with the FDK distance weight.
//
// Filter (mat_codes/filtering.m:5-48, ParkerWeight.m:5-27): the MATLAB code
// zero-pads each detector row to L = max(64, 2^nextpow2(2*nu)), multiplies
// its FFT by the windowed |FFT(ramp)|*2 and crops.  The device does the same
// with its own FFT: two weighted rows travel as the real and imaginary parts
// of one complex signal (the filter response H is real and even, so the two
// filtered rows come back as the real and imaginary parts of the inverse
// transform), forward transform, multiply by H/L, inverse transform as the
// conjugate of a forward transform of the conjugate.  The transforms are
// Stockham autosort FFTs (radix 4, plus one radix-2 stage when log2 L is
// odd) in shared memory; the first stage reads the weighted rows from
// global memory and the last writes the filtered rows.  H is built on the
// host in FP64 (radix-2 FFT below) with the MATLAB scale folded in.
//
// Backprojection (nefct/cc/pixel_3d/pixel.cu.cc:12-146 geometry and index
// rules, Q9-Q11, times (src_iso/(src_iso + x'))^2 from
// mat_codes/backprojection.m:12): one thread owns a column of kZ voxels
// along z; per view it computes the column's rotated position, detector
// column and magnification once and then the kZ row taps (one fused
// multiply-add, an exact floor and four gathers per voxel and view).  Views are
// processed in chunks so a chunk's filtered projections stay in L2.  A
// warp covers an 8 x 4 tile of (x, y) voxel columns.
#include <limits.h>
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

// Transform length of filtering.m: L = max(64, 2^nextpow2(2*nu)).
static int ramp_length(int na)
{
    int p = 0;
    while ((1 << p) < 2 * na) ++p;
    return std::max(64, 1 << p);
}

// H[k] * scale / L for k = 0..L/2 (H[L - k] = H[k]): the windowed filter
// response of filtering.m:54-88 with its scale and the inverse transform's
// 1/L folded in.
static std::vector<float> ramp_response(int na, int window, double scale)
{
    const int L = ramp_length(na);
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
    // Filter (:63-88): 2|FFT|, window on bins 1..L/2 (mirrored to length L)
    std::vector<float> h(L / 2 + 1);
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
        h[k] = (float)(f * scale / L);
    }
    return h;
}

// ---------------- device: weighting + FFT filtering ----------------

static constexpr int kMaxCols = 2048;            // detector columns the filter supports
static constexpr int kMaxL = 4096;               // ramp_length(kMaxCols)
static constexpr int kFftThreads = 256;

struct FilterParams {
    int na, nb, nv, L, log2L, pairs_per_view, pairs;
    float src_det, da, a_shift, db, b_shift;    // cosine weight (FP32)
    double src_det_d, da_d, a_shift_d;          // Parker weight (FP64, as ParkerWeight.m)
    int parker;                                 // 0 off, +1/-1 = ParkerWeight dir
    double dang;                                // view step, degrees
    double fanang;                              // ParkerWeight's fanang (half the fan angle), degrees
    float h[kMaxL / 2 + 1];                     // H[k] * scale / L, k = 0..L/2
};

// Shared-memory index of element e of a transform buffer: C float2 of
// padding per 16 elements.  A stage writes its output with the padding that
// keeps its strided stores free of bank conflicts (fft_cpad) and the next
// stage reads with the same padding; loads of 16 consecutive elements are
// conflict-free under any padding.
template <int C> __host__ __device__ __forceinline__ int fpad(int e) { return e + C * (e >> 4); }

// Padding of the output of the stage with Ns points per finished
// sub-transform: a half-warp writes elements 4j + r (Ns = 1), 8m + k + 2r
// (Ns = 2), 16m + k + 4r (Ns = 4) or 32m + k + 8r (Ns = 8), which C = 1, 2, 4, 4
// spread over 16 distinct 8-byte bank pairs; for Ns >= 16 the half-warp's
// elements are consecutive.
__host__ __device__ constexpr int fft_cpad(int Ns) { return Ns == 1 ? 1 : Ns == 2 ? 2 : Ns <= 8 ? 4 : 1; }

// Shared memory: two padded L-point complex buffers (ping-pong), the
// twiddle tables of the radix-4 stages (stage with Ns points per finished
// sub-transform: W^(r k L/(4 Ns)) at [Ns - 1 or Ns - 2 + (r - 1) Ns + k],
// 3 Ns entries, fewer than L in all) and H[0..L/2].
static constexpr int fft_buf(int L) { return L + L / 4; }   // fpad<4>(L) bound
static inline size_t filt_smem_bytes(int L)
{
    return (size_t)(2 * fft_buf(L) + L) * sizeof(float2) + (size_t)(L / 2 + 4) * sizeof(float);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -(a.y * b.y)), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// (-i) * a
__device__ __forceinline__ float2 cmul_mi(float2 a) { return make_float2(a.y, -a.x); }

// Cosine weight of filtering.m:10, DSD / sqrt(DSD^2 + v^2 + u^2), from the
// row's part c = DSD^2 + v^2 (cos_row) and the column (FP32 with rsqrt: a
// few ulp, against the FP64 of the MATLAB code).
__device__ __forceinline__ float cos_row(const FilterParams &p, int row)
{
    const float v = __fsub_rn(__fmul_rn((float)row + p.b_shift, p.db), __fmul_rn((float)p.nb, p.db) * 0.5f);
    return __fadd_rn(__fmul_rn(p.src_det, p.src_det), __fmul_rn(v, v));
}
__device__ __forceinline__ float cos_weight(const FilterParams &p, float c, int col)
{
    const float u = __fsub_rn(__fmul_rn((float)col + p.a_shift, p.da), __fmul_rn((float)p.na, p.da) * 0.5f);
    return p.src_det * rsqrtf(__fadd_rn(c, __fmul_rn(u, u)));
}

// Parker weight of detector column col at view iv, ParkerWeight.m:5-25
// (1-based views there), in FP64 as the MATLAB code.
__device__ __forceinline__ float parker_weight(const FilterParams &p, int iv, int col)
{
    const double ud = ((double)col + p.a_shift_d) * p.da_d - (double)p.na * p.da_d / 2.0;
    const double as = atan(ud / p.src_det_d) / M_PI * 180.0;
    const double f = p.fanang;
    const double n180 = 180.0 / p.dang;
    const double pw = ((n180 - p.nv) / 2.0 + (iv + 1)) / n180 * 180.0 + p.parker * as;
    double pk = 1.0;
    if (pw <= f / 2 && pw > -f / 2) {
        const double sn = fmax(sin(M_PI / 2 * (f / 2 + pw) / f), 0.0);
        pk = sn * sn;
    }
    if (pw >= 180 - f / 2 && pw < 180 + f / 2) {
        const double c = fmax(cos(M_PI / 2 * (f / 2 + pw - 180) / f), 0.0);
        pk *= c * c;
    }
    if (pw < -f / 2 || pw > 180 + f / 2) pk = 0.0;
    return (float)pk;
}

// One Stockham stage of radix R (2 or 4) of a length-2^LOG2L transform with
// Ns = 2^LNS points per finished sub-transform: butterfly j (< L/R) reads
// elements j + r L/R, multiplies them by W^(r k L/(R Ns)) (k = j mod Ns;
// radix 4 only, from the stage's table tws), transforms them and writes
// them to (j - k) R + k + r Ns.  load(e, i) gives element e (i = fpad(e),
// its shared-memory index); store(e, i, value) takes output element e.  The
// sizes are compile-time, so the index arithmetic folds into constants.
// ZIN: the inputs r >= R/2 are known zero (elements >= L/2 of the padded
// rows in the first stage); LOW: only the outputs r < R/2 are wanted
// (elements < L/2, the cropped rows, in the last stage).
template <int R, int LOG2L, int LNS, int CIN, bool ZIN = false, bool LOW = false, class Load, class Store>
__device__ __forceinline__ void fft_stage(const float2 *tws, Load load, Store store)
{
    constexpr int lR = R == 2 ? 1 : 2;
    constexpr int LR = 1 << (LOG2L - lR), Ns = 1 << LNS;
    constexpr int COUT = fft_cpad(Ns);
    constexpr int PLR = LR + CIN * (LR / 16);          // fpad(j + r LR) = fpad(j) + r PLR (LR % 16 == 0)
    constexpr int ITER = (LR + kFftThreads - 1) / kFftThreads;
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int j = threadIdx.x + it * kFftThreads;
        if (LR % kFftThreads != 0 && j >= LR) break;
        const int k = j & (Ns - 1);
        const int pj = fpad<CIN>(j);
        float2 a[R];
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = (ZIN && r >= R / 2) ? make_float2(0.f, 0.f) : load(j + r * LR, pj + r * PLR);
        const int o = ((j - k) << lR) + k;
        auto out = [&](int r, float2 v) {
            if constexpr (Ns >= 16) store(o + r * Ns, fpad<COUT>(o) + r * (Ns + COUT * (Ns / 16)), v);
            else store(o + r * Ns, fpad<COUT>(o + r * Ns), v);
        };
        if constexpr (R == 2) {
            if constexpr (ZIN) {                 // the radix-2 stage is the first (Ns = 1)
                out(0, a[0]);
                out(1, a[0]);
            } else {
                out(0, cadd(a[0], a[1]));
                out(1, csub(a[0], a[1]));
            }
        } else {
            if constexpr (Ns > 1) {
#pragma unroll
                for (int r = 1; r < 4; ++r)
                    if (!(ZIN && r >= 2)) a[r] = cmul(a[r], tws[(r - 1) * Ns + k]);
            }
            const float2 t0 = ZIN ? a[0] : cadd(a[0], a[2]), t1 = ZIN ? a[0] : csub(a[0], a[2]);
            const float2 t2 = ZIN ? a[1] : cadd(a[1], a[3]), t3 = cmul_mi(ZIN ? a[1] : csub(a[1], a[3]));
            out(0, cadd(t0, t2));
            out(1, cadd(t1, t3));
            if constexpr (!LOW) {
                out(2, csub(t0, t2));
                out(3, csub(t1, t3));
            }
        }
    }
}

// Stages of a length-2^log2L transform: one radix-2 stage first when
// log2L is odd, radix 4 after.
__host__ __device__ constexpr int fft_stages(int log2L) { return (log2L & 1) ? 1 + (log2L - 1) / 2 : log2L / 2; }

// Offset of the twiddle table of the radix-4 stage with Ns points per
// finished sub-transform (Ns = 4^i, or 2 * 4^i after a radix-2 stage).
__host__ __device__ constexpr int tw_offset(int Ns, bool odd) { return odd ? Ns - 2 : Ns - 1; }

// Radix-4 stages from Ns = 2^LNS on: the stages before the last read src
// and write dst in shared memory (swapping them after each stage), the
// last (Ns = L/4) writes through last.
template <int LOG2L, int LNS, bool LOW, class Last>
__device__ __forceinline__ void fft_tail(const float2 *tw, const float2 *src, float2 *dst, Last last)
{
    constexpr bool odd = LOG2L & 1;
    constexpr int CIN = fft_cpad(1 << (LNS - (LNS == 1 ? 1 : 2)));   // the previous stage's output padding
    const float2 *tws = tw + tw_offset(1 << LNS, odd);
    auto ld = [src](int, int i) { return src[i]; };
    if constexpr (LNS + 2 == LOG2L) {
        fft_stage<4, LOG2L, LNS, CIN, false, LOW>(tws, ld, last);
        __syncthreads();
    } else {
        fft_stage<4, LOG2L, LNS, CIN>(tws, ld, [dst](int, int i, float2 v) { dst[i] = v; });
        __syncthreads();
        fft_tail<LOG2L, LNS + 2, LOW>(tw, dst, const_cast<float2 *>(src), last);
    }
}

// Forward FFT of length 2^LOG2L: the first stage reads through first(e, i)
// (ZIN: inputs e >= L/2 are zero), the last writes through last(e, i, value)
// (LOW: outputs e < L/2 only), the stages between ping-pong in shared
// memory (padded indices): stage 0 writes b1, stage 1 b0, ...
template <int LOG2L, bool ZIN, bool LOW, class First, class Last>
__device__ __forceinline__ void fft_run(const float2 *tw, float2 *b0, float2 *b1, First first, Last last)
{
    constexpr bool odd = LOG2L & 1;
    auto to_b1 = [b1](int, int i, float2 v) { b1[i] = v; };
    // the first stage's input index is that of the spectrum buffer (written
    // by a last stage, Ns = L/4 >= 16: padding 1) when it is read from there
    if constexpr (odd) fft_stage<2, LOG2L, 0, 1, ZIN>(tw, first, to_b1);
    else fft_stage<4, LOG2L, 0, 1, ZIN>(tw, first, to_b1);
    __syncthreads();
    fft_tail<LOG2L, odd ? 1 : 2, LOW>(tw, b1, b0, last);
}

// Persistent CTAs over row pairs (view iv, rows b and b + 1); transform
// length 2^LOG2L.
template <int LOG2L>
__global__ void __launch_bounds__(kFftThreads) fdk_filter_kernel(const __grid_constant__ FilterParams p,
                                                                 const float *__restrict__ sino,
                                                                 float *__restrict__ out)
{
    constexpr int L = 1 << LOG2L;
    constexpr bool odd = LOG2L & 1;
    extern __shared__ __align__(16) float2 fsm[];
    const int na = p.na;
    float2 *b0 = fsm, *b1 = fsm + fft_buf(L), *tw = fsm + 2 * fft_buf(L);
    float *hs = reinterpret_cast<float *>(tw + L);
    // twiddle tables of the radix-4 stages: W^(r k L/(4 Ns)) = exp(-2 pi i r k / (4 Ns))
    for (int Ns = odd ? 2 : 1; Ns <= L / 4; Ns *= 4) {
        const int off = tw_offset(Ns, odd);
        for (int i = threadIdx.x; i < 3 * Ns; i += blockDim.x) {
            const int r = 1 + i / Ns, k = i - (r - 1) * Ns;
            float sn, cs;
            sincospif((float)(r * k) / (float)(2 * Ns), &sn, &cs);   // exact argument (power-of-two denominator)
            tw[off + i] = make_float2(cs, -sn);
        }
    }
    for (int k = threadIdx.x; k <= L / 2; k += blockDim.x) hs[k] = p.h[k];
    __syncthreads();
    // the last stage of the forward transform would write b1 after an odd
    // number of stages, b0 after an even number: keep the spectrum there
    float2 *const z = (fft_stages(LOG2L) & 1) ? b1 : b0;
    float2 *const zf = z == b0 ? b1 : b0;
    for (int pr = blockIdx.x; pr < p.pairs; pr += gridDim.x) {
        const int iv = pr / p.pairs_per_view;
        const int row = 2 * (pr - iv * p.pairs_per_view);
        const bool two = row + 1 < p.nb;
        const float *x0 = sino + ((size_t)iv * p.nb + row) * na;
        const float *x1 = x0 + na;
        // forward transform of the weighted pair, zero beyond na
        const float c0 = cos_row(p, row), c1 = cos_row(p, row + 1);
        auto first = [&](int e, int) {
            if (e >= na) return make_float2(0.f, 0.f);
            const float pk = p.parker ? parker_weight(p, iv, e) : 1.f;
            const float a = x0[e] * (cos_weight(p, c0, e) * pk);
            const float b = two ? x1[e] * (cos_weight(p, c1, e) * pk) : 0.f;
            return make_float2(a, b);
        };
        // (rows occupy at most L/2 elements: the upper half of the input is zero)
        fft_run<LOG2L, true, false>(tw, b0, b1, first, [z](int, int i, float2 v) { z[i] = v; });
        // inverse: conj(FFT(conj(Z H / L))); its real and imaginary parts are
        // the filtered rows.  Stage 0 reads z and writes the other buffer,
        // so the second run starts from (z, zf) as (b0, b1).
        auto first2 = [&](int e, int i) {
            const float hk = hs[e <= L / 2 ? e : L - e];
            const float2 v = z[i];
            return make_float2(v.x * hk, -(v.y * hk));
        };
        float *const y0 = out + ((size_t)iv * p.nb + row) * na;
        float *const y1 = y0 + na;
        auto last2 = [&](int e, int, float2 v) {
            if (e < na) {
                y0[e] = v.x;
                if (two) y1[e] = -v.y;
            }
        };
        // (only the first na <= L/2 outputs are kept)
        fft_run<LOG2L, false, true>(tw, z, zf, first2, last2);
    }
}

// Launches the filter for transform length 2^LOG2L.
template <int LOG2L>
static cudaError_t launch_filter(const FilterParams &p, const float *sino, float *out, cudaStream_t s)
{
    const size_t smem = filt_smem_bytes(1 << LOG2L);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(fdk_filter_kernel<LOG2L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fdk_filter_kernel<LOG2L>, kFftThreads, smem);
    const int blocks = std::min(p.pairs, sms * std::max(per_sm, 1));
    fdk_filter_kernel<LOG2L><<<blocks, kFftThreads, smem, s>>>(p, sino, out);
    return cudaGetLastError();
}

// ---------------- device: voxel-driven backprojection ----------------

// Voxels along z per thread: the column part of a view is computed once per
// kZ voxels (measured at 256^3 x 360 views: 2 -> 11.1 ms, 4 -> 8.68 ms,
// 8 -> 8.27 ms, 12 -> 8.47 ms, 16 -> 10.4 ms; 8 holds 61-66 registers
// without spills, more shrink the resident warps).
#ifndef NEFCT_FDK_KZ
#define NEFCT_FDK_KZ 8
#endif
static constexpr int kZ = NEFCT_FDK_KZ;
// Views per launch: as many as fit ~400 MB of a chunk (tap quads: 16 bytes
// per detector cell), 8 to 128.  Fewer launches mean fewer read-modify-write
// passes over the volume and fewer launch tails; that outweighs keeping the
// chunk L2-resident (256^3, 360 views of 512 x 384 with quads: 17 / 32 / 64
// / 128 views per launch take 7.56 / 7.26 / 7.07 / 6.98 ms).
static constexpr int kViewChunk = 128;
static inline int fdk_view_chunk(int na, int nb, size_t bytes_per_cell = sizeof(float))
{
    const double per_view = (double)na * nb * bytes_per_cell;
    return (int)std::min<double>(kViewChunk, std::max<double>(8.0, (double)(400 << 20) / per_view));
}

// Tap quads: for a chunk of views, quad[(v * nb + ib) * na + ia] holds the
// four bilinear taps of detector cell (ia, ib) -- (ia, ib), (ia + 1, ib),
// (ia, ib + 1), (ia + 1, ib + 1) -- so the backprojection reads them with one
// 16-byte load instead of four.  Cells of the last row / column (which the
// backprojection never reads as a quad's origin, Q11) hold zeros.
__global__ void __launch_bounds__(256) fdk_quad_kernel(const float *__restrict__ sino, float4 *__restrict__ quad,
                                                       int na, int nb, long long cells)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cells;
         i += (long long)gridDim.x * blockDim.x) {
        const int ia = (int)(i % na);
        const int ib = (int)((i / na) % nb);
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ia + 1 < na && ib + 1 < nb) {
            const float *s0 = sino + i;
            q = make_float4(__ldg(s0), __ldg(s0 + 1), __ldg(s0 + na), __ldg(s0 + na + 1));
        }
        quad[i] = q;
    }
}
// A warp owns an 8 x 4 (x, y) tile of voxel columns: at any view its
// voxels project onto fewer detector columns than a 32 x 1 row (whose
// detector footprint reaches ~50 columns), so its gathers touch fewer
// sectors (measured 7 % faster than 32 x 1 and 16 x 2, 1 % than 4 x 8).
static constexpr int kTW = 8;

// Voxel centres held in the kernel parameters (x, then y, then z) when the
// three axes together have at most this many voxels.
static constexpr int kCtrMax = 6144;

struct BpParams {
    int nx, ny, nz, na, nb, nv0, nvc, first;
    float sx, sy, sz, corner_x, corner_y, corner_z;
    float src_iso, src_det, da, ai_p, db, bi_p;
    float inv_da, inv_db, cb;         // 1/da, 1/db and nb/2 - bi_p - 0.5, rounded to float
    int cyl, weight;
    float cs[kViewChunk], sn[kViewChunk];
    int has_ctr;                      // ctr holds every voxel centre (else computed per thread)
    float ctr[kCtrMax];
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
// bilinear weights continuously) and floored exactly by the magic-constant
// sum (floor(b) + 1.5*2^23 = round-down(b + 1.5*2^23), valid for |b| < 2^22).
// When |m/db| * max|z| + |nb/2 - bi - 0.5| could reach 2^21 (a voxel at or
// near the source plane has an infinite or NaN b) the thread clamps b to
// [-2, nb + 1] first.  The distance weight is folded into the column
// weights (wa u, wa2 u) once per view.  Every operation is written with its
// rounding (no contraction left to the compiler), so fdk_edge_kernel
// recomputes the same values.
// QUAD: the taps come from the chunk's tap quads (fdk_quad_kernel) with one
// 16-byte load; the arithmetic is the same, so are the results, bit for bit.

// Column part of one view for the voxel column at (xc, yc): bp_column the
// detector column (a, ia) and the magnification, bp_weights (for a column
// that is kept) the row slope bm and the column weights.
struct BpColumn {
    float a, bm, wau, wa2u;
    float inv, m;
    int ia;
};

__device__ __forceinline__ void bp_column(const BpParams &p, float cphi, float sphi, float xc, float yc, BpColumn &c)
{
    const float xc0 = __fmaf_rn(xc, cphi, __fmul_rn(yc, sphi));
    const float yc0 = __fmaf_rn(-xc, sphi, __fmul_rn(yc, cphi));
    const float nah = (float)(p.na / 2);                   // integer half (Q9)
    // 1 / (xc0 - xs) = 1 / (src_iso + xc0): magnification and distance weight share it
    c.inv = rcp_approx(__fadd_rn(xc0, p.src_iso));
    c.m = __fmul_rn(p.src_det, c.inv);                     // SAD / (xc0 - xs)
    float t;
    if (p.cyl) t = __fmaf_rn(atan2f(yc0, __fadd_rn(xc0, p.src_iso)), p.inv_da, nah);
    else t = __fmaf_rn(__fmul_rn(c.m, yc0), p.inv_da, nah);
    c.a = __fsub_rn(__fsub_rn(t, p.ai_p), 0.5f);
    c.ia = __float2int_rd(c.a);
}

__device__ __forceinline__ void bp_weights(const BpParams &p, BpColumn &c)
{
    c.bm = __fmul_rn(c.m, p.inv_db);
    float u = 1.f;
    if (p.weight) {
        const float r = __fmul_rn(p.src_iso, c.inv);
        u = __fmul_rn(r, r);
    }
    const float wa2 = __fsub_rn(c.a, (float)c.ia), wa = __fsub_rn(1.f, wa2);
    c.wau = __fmul_rn(wa, u);
    c.wa2u = __fmul_rn(wa2, u);
}

// Voxel centre along one axis, pixel.cu.cc:116-118 ((i + 0.5) * s / n + c, in double).
__host__ __device__ __forceinline__ float bp_centre(int i, float s, int n, float c)
{
    return (float)((i + 0.5) * (double)s / n + (double)c);
}
// The same from the host-filled table (the host's double arithmetic gives
// the same values), saving each thread its double divisions per launch.
__device__ __forceinline__ float bp_cx(const BpParams &p, int i)
{
    return p.has_ctr ? p.ctr[i] : bp_centre(i, p.sx, p.nx, p.corner_x);
}
__device__ __forceinline__ float bp_cy(const BpParams &p, int i)
{
    return p.has_ctr ? p.ctr[p.nx + i] : bp_centre(i, p.sy, p.ny, p.corner_y);
}
__device__ __forceinline__ float bp_cz(const BpParams &p, int i)
{
    return p.has_ctr ? p.ctr[p.nx + p.ny + i] : bp_centre(i, p.sz, p.nz, p.corner_z);
}

// Contribution of one voxel at detector row b from the column's taps:
// false when Q11 drops it (ib < 0 || ib + 1 >= nb).
template <bool QUAD>
__device__ __forceinline__ bool bp_tap(const BpParams &p, const float *pv, const float4 *pq, const BpColumn &c, float b,
                                       float &r0, float &r1, float &wb, float &wb2)
{
    const float mb = __fadd_rd(b, 12582912.0f);
    const unsigned ib = (unsigned)(__float_as_int(mb) - 0x4B400000);
    if (ib >= (unsigned)(p.nb - 1)) return false;
    wb2 = __fsub_rn(b, __fsub_rn(mb, 12582912.0f));
    wb = __fsub_rn(1.f, wb2);
    float t00, t01, t10, t11;
    if (QUAD) {
        const float4 q4 = __ldg(pq + (size_t)ib * p.na);
        t00 = q4.x; t01 = q4.y; t10 = q4.z; t11 = q4.w;
    } else {
        const float *q = pv + (size_t)ib * p.na;
        t00 = __ldg(q); t01 = __ldg(q + 1); t10 = __ldg(q + p.na); t11 = __ldg(q + p.na + 1);
    }
    r0 = __fmaf_rn(t01, c.wa2u, __fmul_rn(t00, c.wau));
    r1 = __fmaf_rn(t11, c.wa2u, __fmul_rn(t10, c.wau));
    return true;
}

template <bool QUAD>
__global__ void __launch_bounds__(128) fdk_bp_kernel(const __grid_constant__ BpParams p,
                                                     const float *__restrict__ sino, const float4 *__restrict__ quad,
                                                     float *__restrict__ vol)
{
    const int ix = blockIdx.x * kTW + (threadIdx.x % kTW);
    const int iy = (blockIdx.y * 4 + threadIdx.y) * (32 / kTW) + threadIdx.x / kTW;
    const int z0 = blockIdx.z * kZ;
    if (ix >= p.nx || iy >= p.ny) return;
    const float xc = bp_cx(p, ix);
    const float yc = bp_cy(p, iy);
    float zc[kZ], acc[kZ];
    const size_t plane = (size_t)p.nx * p.ny;
    const size_t col = (size_t)iy * p.nx + ix;
#pragma unroll
    for (int k = 0; k < kZ; ++k) {
        const int iz = z0 + k;
        zc[k] = bp_cz(p, min(iz, p.nz - 1));
        acc[k] = (!p.first && iz < p.nz) ? vol[iz * plane + col] : 0.f;
    }
    float zabs = 0.f;
#pragma unroll
    for (int k = 0; k < kZ; ++k) zabs = fmaxf(zabs, fabsf(zc[k]));
    const float bhi = (float)(p.nb + 1);
    for (int v = 0; v < p.nvc; ++v) {
        BpColumn c;
        bp_column(p, p.cs[v], p.sn[v], xc, yc, c);
        if (c.ia < 0 || c.ia + 1 >= p.na) continue;             // Q11
        bp_weights(p, c);
        const float *pv = sino + (size_t)v * p.na * p.nb + c.ia;
        const float4 *pq = QUAD ? quad + (size_t)v * p.na * p.nb + c.ia : nullptr;
        float r0, r1, wb, wb2;
        if (fabsf(c.bm) * zabs + fabsf(p.cb) < 2097152.f) {
#pragma unroll
            for (int k = 0; k < kZ; ++k) {
                // branch-free: a dropped row (Q11) reads row nb - 2's taps with
                // zero weights (adds +0: measured 2.6 % faster than skipping)
                const float b = __fmaf_rn(c.bm, zc[k], p.cb);
                const float mb = __fadd_rd(b, 12582912.0f);
                const unsigned ib = (unsigned)(__float_as_int(mb) - 0x4B400000);
                const bool keep = ib < (unsigned)(p.nb - 1);
                const unsigned ibc = keep ? ib : (unsigned)(p.nb - 2);
                const float w2 = __fsub_rn(b, __fsub_rn(mb, 12582912.0f));
                const float wb2k = keep ? w2 : 0.f, wbk = keep ? __fsub_rn(1.f, w2) : 0.f;
                float t00, t01, t10, t11;
                if (QUAD) {
                    const float4 q4 = __ldg(pq + (size_t)ibc * p.na);
                    t00 = q4.x; t01 = q4.y; t10 = q4.z; t11 = q4.w;
                } else {
                    const float *q = pv + (size_t)ibc * p.na;
                    t00 = __ldg(q); t01 = __ldg(q + 1); t10 = __ldg(q + p.na); t11 = __ldg(q + p.na + 1);
                }
                const float a0 = __fmaf_rn(t01, c.wa2u, __fmul_rn(t00, c.wau));
                const float a1 = __fmaf_rn(t11, c.wa2u, __fmul_rn(t10, c.wau));
                acc[k] = __fmaf_rn(a1, wb2k, __fmaf_rn(a0, wbk, acc[k]));
            }
        } else {
#pragma unroll
            for (int k = 0; k < kZ; ++k)
                if (bp_tap<QUAD>(p, pv, pq, c, fminf(fmaxf(__fmaf_rn(c.bm, zc[k], p.cb), -2.f), bhi), r0, r1, wb, wb2))
                    acc[k] = __fmaf_rn(r1, wb2, __fmaf_rn(r0, wb, acc[k]));
        }
    }
#pragma unroll
    for (int k = 0; k < kZ; ++k)
        if (z0 + k < p.nz) vol[(z0 + k) * plane + col] = acc[k];
}

// ---- detector-edge decisions with the reference's own operations ----
//
// The few-ulp differences above move the bilinear weights continuously
// everywhere except at the detector's edges, where the reference drops a
// voxel whose tap pair reaches past the last column or row, or starts before
// the first (Q11): there a row or column within ulps of the edge can be kept
// by one evaluation and dropped by the other.  For a flat detector,
// fdk_edge_kernel revisits, after fdk_bp_kernel, every (column, view) of the
// chunk whose detector column lies within `edge` of column 0 or na - 1, and
// every voxel whose row lies within `edge` of row 0 or nb - 1; it decides
// each with the reference's operations in order (pixel.cu.cc:24-33, no
// contraction: exact_col, exact_row) and takes a voxel the kernel kept and
// the reference drops out of the sum, or puts one the reference keeps in.

// pixel.cu.cc:24-29: the rotated voxel centre and the magnification
// SAD / (x' - xs) (xs = -src_iso).
__device__ __forceinline__ float exact_mag(const BpParams &p, float cphi, float sphi, float xc, float yc, float &yr)
{
    const float xr = __fadd_rn(__fmul_rn(xc, cphi), __fmul_rn(yc, sphi));
    yr = __fadd_rn(__fmul_rn(-xc, sphi), __fmul_rn(yc, cphi));
    return __fdiv_rn(p.src_det, __fadd_rn(xr, p.src_iso));
}

// pixel.cu.cc:30-32: a = yd / da + na / 2 - ai - 0.5 (the last subtraction
// in double, rounded to float: the same as the float subtraction).
__device__ __forceinline__ float exact_col(const BpParams &p, float cphi, float sphi, float xc, float yc)
{
    float yr;
    const float m = exact_mag(p, cphi, sphi, xc, yc, yr);
    return __fsub_rn(__fsub_rn(__fadd_rn(__fdiv_rn(__fmul_rn(m, yr), p.da), (float)(p.na / 2)), p.ai_p), 0.5f);
}

// pixel.cu.cc:28,31: b = (SAD / (x' - xs)) * z / db + nb / 2 - bi - 0.5.
__device__ __forceinline__ float exact_row(const BpParams &p, float cphi, float sphi, float xc, float yc, float zc)
{
    float yr;
    const float m = exact_mag(p, cphi, sphi, xc, yc, yr);
    return __fsub_rn(__fsub_rn(__fadd_rn(__fdiv_rn(__fmul_rn(m, zc), p.db), (float)(p.nb / 2)), p.bi_p), 0.5f);
}

// Column (row) decisions: kept when 0 <= floor(x) and floor(x) + 1 < n.
__device__ __forceinline__ bool bp_keep(float x, int n)
{
    const int i = __float2int_rd(x);
    return i >= 0 && i + 1 < n;
}

// One warp per voxel column; lane l takes views l, l + 32, ... of one table
// (up to kViewChunk views, after every chunk's backprojection) and finds, in
// parallel, the voxels whose decisions differ and the corrections; the
// corrections are then applied by one lane at a time in view order, so the
// result stays deterministic (and the same with and without tap quads: the
// taps are read from the filtered sinogram, which the quads copy).
static constexpr int kEdgeSlots = 4;

__global__ void __launch_bounds__(256) fdk_edge_kernel(const __grid_constant__ BpParams p,
                                                       const float *__restrict__ sino, float *vol)
{
    // the view table in shared memory: lanes read different views, which the
    // parameter bank would serve one address at a time
    __shared__ float s_cs[kViewChunk], s_sn[kViewChunk];
    for (int i = threadIdx.x; i < p.nvc; i += blockDim.x) {
        s_cs[i] = p.cs[i];
        s_sn[i] = p.sn[i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long colid = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (colid >= (long long)p.nx * p.ny) return;           // uniform across the warp
    const int ix = (int)(colid % p.nx), iy = (int)(colid / p.nx);
    const float xc = bp_cx(p, ix);
    const float yc = bp_cy(p, iy);
    const float naf = (float)p.na, nbf = (float)p.nb;
    // Width of the bands decided again: the kernel's detector coordinate
    // differs from the reference's by a few ulp of terms of about half the
    // detector (rcp_approx and the fused row: <= ~8 ulp of max(na, nb), i.e.
    // under max(na, nb) * 2^-20); the band is 16x that plus 1/1024.  A
    // wider band only adds work (every voxel in it is decided twice).
    const float edge = 1.f / 1024 + fmaxf(naf, nbf) * (1.f / 65536);
    const size_t plane = (size_t)p.nx * p.ny;
    float *const vcol = vol + (size_t)iy * p.nx + ix;
    const float idz = (float)p.nz / p.sz;
    const float z_first = bp_cz(p, 0), z_last = bp_cz(p, p.nz - 1);
    for (int v0 = 0; v0 < p.nvc; v0 += 32) {
        const int v = v0 + lane;
        const bool has = v < p.nvc;
        const int vt = min(v, p.nvc - 1);                  // lanes past the table read its last entry
        const float cphi = s_cs[vt], sphi = s_sn[vt];
        BpColumn c, cr;
        bool col_ours = false, col_ref = false;
        if (has) {
            bp_column(p, cphi, sphi, xc, yc, c);
            bp_weights(p, c);
            col_ours = c.ia >= 0 && c.ia + 1 < p.na;
            col_ref = col_ours;
            cr = c;                           // the column as the reference places it
            if (!p.cyl && (fabsf(c.a) < edge || fabsf(c.a - (naf - 1.f)) < edge)) {
                cr.a = exact_col(p, cphi, sphi, xc, yc);
                cr.ia = __float2int_rd(cr.a);
                col_ref = cr.ia >= 0 && cr.ia + 1 < p.na;
                const float wa2 = __fsub_rn(cr.a, (float)cr.ia);
                const float u = __fadd_rn(c.wau, c.wa2u);     // the distance weight (wa + wa2 = 1)
                cr.wau = __fmul_rn(__fsub_rn(1.f, wa2), u);
                cr.wa2u = __fmul_rn(wa2, u);
            }
        }
        const size_t off = (size_t)v * p.na * p.nb;
        auto contribution = [&](const BpColumn &cc, float b, float &out) -> bool {
            float r0, r1, wb, wb2;
            if (!bp_tap<false>(p, sino + off + cc.ia, nullptr, cc, b, r0, r1, wb, wb2)) return false;
            out = __fmaf_rn(r1, wb2, __fmul_rn(r0, wb));
            return true;
        };
        // correction of voxel iz (0 where the decisions agree)
        auto delta = [&](int iz, bool whole_column) -> float {
            const float zc = bp_cz(p, iz);
            const float b = __fmaf_rn(c.bm, zc, p.cb);
            const bool near_row = fabsf(b) < edge || fabsf(b - (nbf - 1.f)) < edge;
            if (!whole_column && !near_row) return 0.f;
            const float br = near_row ? exact_row(p, cphi, sphi, xc, yc, zc) : b;
            float co = 0.f, cref = 0.f;
            const bool ours = col_ours && bp_keep(b, p.nb) && contribution(c, b, co);
            const bool ref = col_ref && bp_keep(br, p.nb) && contribution(cr, br, cref);
            if (ours == ref && !whole_column) return 0.f;
            return __fsub_rn(ref ? cref : 0.f, ours ? co : 0.f);
        };
        // voxel range of the band of rows within `edge` of row 0 (e = 0) or
        // nb - 1 (e = 1): the rows are monotone in z (b = bm z + cb), so the
        // band is one z interval, mapped to voxel indices in float with a
        // margin of 1/1024 voxel (its rounding is ~1e-5 voxel); the band is
        // a few thousandths of a voxel wide, so few (column, view) pairs have
        // a candidate and few warps take the (divergent) candidate path
        float b_first = 0.f, b_last = 0.f, ibm = 0.f;
        auto band = [&](int e, int &i0, int &i1) {
            const float target = e ? nbf - 1.f : 0.f;
            const float za = (target - edge - p.cb) * ibm, zb = (target + edge - p.cb) * ibm;
            const float flo = (fminf(za, zb) - p.corner_z) * idz - 0.5f - 1.f / 1024;
            const float fhi = (fmaxf(za, zb) - p.corner_z) * idz - 0.5f + 1.f / 1024;
            i0 = max(0, __float2int_ru(fmaxf(flo, -1.f)));
            i1 = min(p.nz - 1, __float2int_rd(fminf(fhi, (float)p.nz)));
        };
        // rows of the column over the grid's z extent (a little wider): a
        // band outside it has no voxel
        auto reaches = [&](int e) {
            const float target = e ? nbf - 1.f : 0.f;
            return fminf(b_first, b_last) - 1.f < target && target < fmaxf(b_first, b_last) + 1.f;
        };
        int n = 0, slot_iz[kEdgeSlots];
        float slot_d[kEdgeSlots];
        bool serial = has && col_ours != col_ref;   // the whole column differs: done one lane at a time
        if (has && !serial && col_ours && c.bm != 0.f) {
            b_first = __fmaf_rn(c.bm, z_first, p.cb);
            b_last = __fmaf_rn(c.bm, z_last, p.cb);
            ibm = rcp_approx(c.bm);
            for (int e = 0; e < 2; ++e) {
                if (!reaches(e)) continue;
                int i0, i1;
                band(e, i0, i1);
                for (int iz = i0; iz <= i1; ++iz) {
                    const float d = delta(iz, false);
                    if (d == 0.f) continue;
                    if (n < kEdgeSlots) { slot_iz[n] = iz; slot_d[n] = d; ++n; }
                    else serial = true;
                }
            }
        }
        // apply in view order: lane by lane
        unsigned pending = __ballot_sync(0xffffffffu, n > 0 || serial);
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1;
            if (lane == src) {
                if (col_ours != col_ref) {
                    for (int iz = 0; iz < p.nz; ++iz) {
                        const float d = delta(iz, true);
                        if (d != 0.f) vcol[(size_t)iz * plane] = __fadd_rn(vcol[(size_t)iz * plane], d);
                    }
                } else if (serial) {                   // more corrections than slots (rare)
                    for (int e = 0; e < 2; ++e) {
                        int i0, i1;
                        band(e, i0, i1);
                        for (int iz = i0; iz <= i1; ++iz) {
                            const float d = delta(iz, false);
                            if (d != 0.f) vcol[(size_t)iz * plane] = __fadd_rn(vcol[(size_t)iz * plane], d);
                        }
                    }
                } else {
                    for (int k = 0; k < n; ++k)
                        vcol[(size_t)slot_iz[k] * plane] = __fadd_rn(vcol[(size_t)slot_iz[k] * plane], slot_d[k]);
                }
            }
            __syncwarp();
        }
    }
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
    p.L = ramp_length(g->na);
    p.log2L = 0;
    while ((1 << p.log2L) < p.L) ++p.log2L;
    p.pairs_per_view = (g->nb + 1) / 2;
    if ((long long)p.pairs_per_view * g->nv > INT_MAX) { delete pp; return fail(NEFCT_ERR_UNSUPPORTED, "too many detector rows x views"); }
    p.pairs = p.pairs_per_view * g->nv;
    p.src_det = g->src_det; p.da = g->da; p.a_shift = g->a_shift; p.db = g->db; p.b_shift = g->b_shift;
    p.src_det_d = g->src_det; p.da_d = g->da; p.a_shift_d = g->a_shift;
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
    const std::vector<float> h = ramp_response(g->na, window, scale);
    std::copy(h.begin(), h.end(), p.h);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if (p.pairs > 0) {
        switch (p.log2L) {
        case 6: e = launch_filter<6>(p, sino, out, s); break;
        case 7: e = launch_filter<7>(p, sino, out, s); break;
        case 8: e = launch_filter<8>(p, sino, out, s); break;
        case 9: e = launch_filter<9>(p, sino, out, s); break;
        case 10: e = launch_filter<10>(p, sino, out, s); break;
        case 11: e = launch_filter<11>(p, sino, out, s); break;
        case 12: e = launch_filter<12>(p, sino, out, s); break;
        default: delete pp; return fail(NEFCT_ERR_UNSUPPORTED, "FFT length 2^%d outside 2^6..2^12", p.log2L);
        }
    }
    if (e != cudaSuccess) { delete pp; return cuda_fail(e, "fdk_filter_kernel"); }
    delete pp;
    NEFCT_CHECK_LAUNCH("fdk_filter_kernel");
    return NEFCT_OK;
}

size_t nefct_fdk_workspace_bytes(const nefct_cb_geom *g)
{
    if (!g || g->na < 1 || g->nb < 1) return 0;
    const int chunk = fdk_view_chunk(g->na, g->nb, sizeof(float4));
    return (size_t)std::min(chunk, std::max(g->nv, 1)) * g->na * g->nb * sizeof(float4);
}

nefct_status nefct_fdk_backproject_ws(const nefct_cb_geom *g, const float *filtered, float *vol, uint32_t flags,
                                      void *ws, size_t ws_bytes, void *stream)
{
    nefct_status st = check_cb_geom(g);
    if (st) return st;
    if (!filtered || !vol) return fail(NEFCT_ERR_INVALID, "filtered and vol must be non-NULL");
    if (flags & ~NEFCT_FDK_NO_WEIGHT) return fail(NEFCT_ERR_INVALID, "unknown flag bits 0x%x", flags);
    const bool quad = ws != nullptr;
    if (quad && ws_bytes < nefct_fdk_workspace_bytes(g))
        return fail(NEFCT_ERR_WORKSPACE, "needs %zu workspace bytes, got %zu", nefct_fdk_workspace_bytes(g), ws_bytes);
    if (quad && ((uintptr_t)ws & 15)) return fail(NEFCT_ERR_INVALID, "workspace must be 16-byte aligned");
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
    p->has_ctr = (long long)g->grid.nx + g->grid.ny + g->grid.nz <= kCtrMax;
    if (p->has_ctr) {
        float *c = p->ctr;
        for (int i = 0; i < p->nx; ++i) *c++ = bp_centre(i, p->sx, p->nx, p->corner_x);
        for (int i = 0; i < p->ny; ++i) *c++ = bp_centre(i, p->sy, p->ny, p->corner_y);
        for (int i = 0; i < p->nz; ++i) *c++ = bp_centre(i, p->sz, p->nz, p->corner_z);
    }
    cudaStream_t s = (cudaStream_t)stream;
    dim3 grid((g->grid.nx + kTW - 1) / kTW, (g->grid.ny + 4 * (32 / kTW) - 1) / (4 * (32 / kTW)), (g->grid.nz + kZ - 1) / kZ);
    const int chunk = quad ? fdk_view_chunk(g->na, g->nb, sizeof(float4)) : fdk_view_chunk(g->na, g->nb);
    float4 *q4 = (float4 *)ws;
    for (int v0 = 0; v0 < g->nv; v0 += chunk) {
        p->nv0 = v0;
        p->nvc = std::min(chunk, g->nv - v0);
        p->first = v0 == 0;
        for (int i = 0; i < p->nvc; ++i) {
            p->cs[i] = (float)cos((double)g->angles[v0 + i]);
            p->sn[i] = (float)sin((double)g->angles[v0 + i]);
        }
        const float *chunk_sino = filtered + (size_t)v0 * g->na * g->nb;
        cudaError_t e;
        if (quad) {
            const long long cells = (long long)p->nvc * g->na * g->nb;
            const unsigned blocks = (unsigned)std::min<long long>((cells + 255) / 256, 148ll * 16);
            fdk_quad_kernel<<<blocks, 256, 0, s>>>(chunk_sino, q4, g->na, g->nb, cells);
            e = cudaGetLastError();
            if (e != cudaSuccess) { delete p; return cuda_fail(e, "fdk_quad_kernel"); }
            fdk_bp_kernel<true><<<grid, dim3(32, 4), 0, s>>>(*p, chunk_sino, q4, vol);
        } else {
            fdk_bp_kernel<false><<<grid, dim3(32, 4), 0, s>>>(*p, chunk_sino, nullptr, vol);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) { delete p; return cuda_fail(e, "fdk_bp_kernel"); }
    }
    // detector-edge decisions, a warp per voxel column, kViewChunk views per launch
    const long long columns = (long long)g->grid.nx * g->grid.ny;
    const unsigned eblocks = (unsigned)((columns + 7) / 8);        // a warp per column
    for (int v0 = 0; v0 < g->nv; v0 += kViewChunk) {
        p->nv0 = v0;
        p->nvc = std::min(kViewChunk, g->nv - v0);
        for (int i = 0; i < p->nvc; ++i) {
            p->cs[i] = (float)cos((double)g->angles[v0 + i]);
            p->sn[i] = (float)sin((double)g->angles[v0 + i]);
        }
        fdk_edge_kernel<<<eblocks, 256, 0, s>>>(*p, filtered + (size_t)v0 * g->na * g->nb, vol);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { delete p; return cuda_fail(e, "fdk_edge_kernel"); }
    }
    delete p;
    return NEFCT_OK;
}

nefct_status nefct_fdk_backproject(const nefct_cb_geom *g, const float *filtered, float *vol, uint32_t flags,
                                   void *stream)
{
    return nefct_fdk_backproject_ws(g, filtered, vol, flags, nullptr, 0, stream);
}

}  // extern "C"
