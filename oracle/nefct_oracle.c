/*
 * TEST INFRASTRUCTURE (oracle).  CPU restatement of the reference's
 * projector hot path; see nefct_oracle.h.  Only tests/, the smoke check and
 * the benchmark's CPU-baseline leg may load this library.
 *
 * Build: oracle/Makefile (gcc -O3 -fopenmp -ffp-contract=off).  Contraction
 * is off so that float results follow the reference's evaluation order.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "nefct_oracle.h"

/* Deterministic scatters split their rows into this many chunks, whatever the
 * thread count (the reference build's shim uses the same number). */
#define OR_CHUNKS 16

/* ---- slab walk, cone-beam and LOR drivers: float and double builds ---- */
#define REAL float
#define SUF _f32
#define SQRT sqrtf
#define FLOOR floorf
#define COS cosf
#define SIN sinf
#include "walk.inc"
#undef REAL
#undef SUF
#undef SQRT
#undef FLOOR
#undef COS
#undef SIN

#define REAL double
#define SUF _f64
#define SQRT sqrt
#define FLOOR floor
#define COS cos
#define SIN sin
#include "walk.inc"
#undef REAL
#undef SUF
#undef SQRT
#undef FLOOR
#undef COS
#undef SIN

void or_trig_f32(const float *angles, int nv, int use_cosf, float *cs, float *sn)
{
    for (int i = 0; i < nv; ++i) {
        if (use_cosf) { cs[i] = cosf(angles[i]); sn[i] = sinf(angles[i]); }
        else { cs[i] = (float)cos((double)angles[i]); sn[i] = (float)sin((double)angles[i]); }
    }
}

/* ---- exact FP64 radiological path ----
 * Plane-crossing parametrisation of the segment p1->p2 (Siddon 1985,
 * Jacobs et al. 1998): collect the alpha of every grid plane the segment
 * crosses inside the volume, sort, and sum f(voxel at segment midpoint) *
 * (alpha_{k+1} - alpha_k) * |p2 - p1|. */
static int cmp_double(const void *a, const void *b)
{
    const double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

static double exact_ray(const or_grid *g, const double *img, const double p1[3], const double p2[3],
                        double *buf)
{
    const int n[3] = {g->nx, g->ny, g->nz};
    const double c[3] = {g->cx, g->cy, g->cz}, s[3] = {g->sx, g->sy, g->sz};
    double lo[3], d[3], dir[3];
    double amin = 0.0, amax = 1.0;
    for (int k = 0; k < 3; ++k) {
        lo[k] = c[k] - s[k] / 2.0;
        d[k] = s[k] / n[k];
        dir[k] = p2[k] - p1[k];
        if (dir[k] != 0.0) {
            double a0 = (lo[k] - p1[k]) / dir[k], a1 = (lo[k] + s[k] - p1[k]) / dir[k];
            if (a0 > a1) { double t = a0; a0 = a1; a1 = t; }
            if (a0 > amin) amin = a0;
            if (a1 < amax) amax = a1;
        } else if (p1[k] < lo[k] || p1[k] >= lo[k] + s[k]) {
            return 0.0;
        }
    }
    if (amax <= amin) return 0.0;
    int m = 0;
    buf[m++] = amin;
    for (int k = 0; k < 3; ++k) {
        if (dir[k] == 0.0) continue;
        for (int i = 0; i <= n[k]; ++i) {
            const double a = (lo[k] + i * d[k] - p1[k]) / dir[k];
            if (a > amin && a < amax) buf[m++] = a;
        }
    }
    buf[m++] = amax;
    qsort(buf, (size_t)m, sizeof(double), cmp_double);
    const double len = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    double acc = 0.0;
    for (int j = 0; j + 1 < m; ++j) {
        const double da = buf[j + 1] - buf[j];
        if (da <= 0.0) continue;
        const double am = 0.5 * (buf[j] + buf[j + 1]);
        int id[3];
        int ok = 1;
        for (int k = 0; k < 3; ++k) {
            id[k] = (int)floor((p1[k] + am * dir[k] - lo[k]) / d[k]);
            if (id[k] < 0 || id[k] >= n[k]) ok = 0;
        }
        if (ok) acc += img[id[0] + (long long)id[1] * n[0] + (long long)id[2] * n[0] * n[1]] * da * len;
    }
    return acc;
}

void or_cb_exact_f64(const or_grid *g, const double *img, const double *angles, const double *off,
                     int nv, double src_iso, double src_det, int na, double da, double ai,
                     int nb, double db, double bi, int cyl, int inv_l2, double *sino)
{
    const double dxp = (double)g->sx / g->nx;
    const int cap = g->nx + g->ny + g->nz + 8;
    #pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * (size_t)cap);
        #pragma omp for schedule(dynamic, 1)
        for (int iv = 0; iv < nv; ++iv) {
            const double cs = cos(angles[iv]), sn = sin(angles[iv]);
            const double o = off ? off[iv] : 0.0;
            for (int ib = 0; ib < nb; ++ib)
                for (int ia = 0; ia < na; ++ia) {
                    double p[6];
                    or_cb_ray_f64(cs, sn, o, ia, ib, na, nb, src_iso, src_det, da, ai, db, bi, cyl, p);
                    double v = exact_ray(g, img, p, p + 3, buf);
                    if (inv_l2) {
                        const double dx = p[3] - p[0], dy = p[4] - p[1], dz = p[5] - p[2];
                        v /= (dx * dx + dy * dy + dz * dz) / (dxp * dxp);
                    }
                    sino[(long long)iv * na * nb + (long long)ib * na + ia] = v;
                }
        }
        free(buf);
    }
}

/* ---- voxel-driven bilinear backprojection, pixel.cu.cc:12-146 ----
 * Written once for float and once for double in the reference's order:
 * voxel centre (ix + 0.5)*sx/nx + cx in double then rounded (:116-118),
 * detector index yd/da + na/2 - ai - 0.5 with integer na/2 (Q9), taps
 * skipped when ia+1 >= na or ib+1 >= nb (Q11). */
#define PIXEL_BODY(REAL, COSF, SINF, ATAN2F, FLOORF)                                            \
    _Pragma("omp parallel for collapse(2) schedule(static)")                                      \
    for (int iz = 0; iz < nz; ++iz)                                                                \
        for (int iy = 0; iy < ny; ++iy)                                                            \
            for (int ix = 0; ix < nx; ++ix) {                                                      \
                const REAL xc = (REAL)((ix + 0.5) * size[0] / nx + corner[0]);                     \
                const REAL yc = (REAL)((iy + 0.5) * size[1] / ny + corner[1]);                     \
                const REAL zc = (REAL)((iz + 0.5) * size[2] / nz + corner[2]);                     \
                const REAL xs = -src_iso;                                                          \
                REAL acc = (REAL)0;                                                                \
                for (int iv = 0; iv < nv; ++iv) {                                                  \
                    const REAL cphi = COSF(angles[iv]), sphi = SINF(angles[iv]);                   \
                    const REAL xc0 = xc * cphi + yc * sphi;                                        \
                    const REAL yc0 = -xc * sphi + yc * cphi;                                       \
                    REAL t;                                                                        \
                    if (cyl) {                                                                     \
                        const REAL ang = ATAN2F(yc0, xc0 + src_iso);                               \
                        t = ang / da + (REAL)(na / 2);                                             \
                    } else {                                                                       \
                        const REAL yd = src_det / (xc0 - xs) * yc0;                                \
                        t = yd / da + (REAL)(na / 2);                                              \
                    }                                                                              \
                    t = t - ai;                                                                    \
                    const REAL a = (REAL)((double)t - 0.5);                                        \
                    const REAL zd = src_det / (xc0 - xs) * zc;                                     \
                    REAL tb = zd / db + (REAL)(nb / 2);                                            \
                    tb = tb - bi;                                                                  \
                    const REAL b = (REAL)((double)tb - 0.5);                                       \
                    const int ia = (int)FLOORF(a), ia2 = ia + 1;                                   \
                    const int ib = (int)FLOORF(b), ib2 = ib + 1;                                   \
                    const REAL wa2 = a - (REAL)ia, wa = (REAL)1 - wa2;                             \
                    const REAL wb2 = b - (REAL)ib, wb = (REAL)1 - wb2;                             \
                    if (ia < 0 || ia2 >= na) continue;                                             \
                    if (ib < 0 || ib2 >= nb) continue;                                             \
                    const REAL *p = sino + (long long)iv * na * nb;                                \
                    REAL s = p[ia + ib * na] * wa * wb + p[ia + ib2 * na] * wa * wb2 +             \
                             p[ia2 + ib * na] * wa2 * wb + p[ia2 + ib2 * na] * wa2 * wb2;          \
                    if (fdk) {                                                                     \
                        const REAL r = src_iso / (src_iso + xc0);                                  \
                        s = s * (r * r);                                                           \
                    }                                                                              \
                    acc += s;                                                                      \
                }                                                                                  \
                img[ix + (long long)iy * nx + (long long)iz * nx * ny] = acc;                      \
            }

void or_pixel_backproject_f32(const float *sino, const float *angles, int nv,
                              int nx, int ny, int nz, const float *corner, const float *size,
                              float src_iso, float src_det, int na, float da, float ai,
                              int nb, float db, float bi, int cyl, int fdk, float *img)
{
    PIXEL_BODY(float, cosf, sinf, atan2f, floorf)
}

void or_pixel_backproject_f64(const double *sino, const double *angles, int nv,
                              int nx, int ny, int nz, const double *corner, const double *size,
                              double src_iso, double src_det, int na, double da, double ai,
                              int nb, double db, double bi, int cyl, int fdk, double *img)
{
    PIXEL_BODY(double, cos, sin, atan2, floor)
}

/* ---- trilinear warp, cpp/deform/deform.cu.cc:13-46 ---- */
#define DEFORM_BODY(REAL, FLOORF)                                                                 \
    _Pragma("omp parallel for collapse(2) schedule(static)")                                      \
    for (int iz = 0; iz < nz; ++iz)                                                                \
        for (int iy = 0; iy < ny; ++iy)                                                            \
            for (int ix = 0; ix < nx; ++ix) {                                                      \
                const long long id = ix + (long long)iy * nx + (long long)iz * nx * ny;            \
                const long long sy = nx, sz = (long long)nx * ny;                                  \
                const REAL px = (REAL)ix + mx[id], py = (REAL)iy + my[id], pz = (REAL)iz + mz[id]; \
                const int xi = (int)FLOORF(px), yi = (int)FLOORF(py), zi = (int)FLOORF(pz);        \
                out[id] = (REAL)0;                                                                 \
                /* Q13: base index 0 is rejected as well as out-of-range ones */                   \
                if (xi <= 0 || xi + 1 >= nx || yi <= 0 || yi + 1 >= ny || zi <= 0 || zi + 1 >= nz) \
                    continue;                                                                      \
                const REAL wx2 = px - (REAL)xi, wx = (REAL)1 - wx2;                                \
                const REAL wy2 = py - (REAL)yi, wy = (REAL)1 - wy2;                                \
                const REAL wz2 = pz - (REAL)zi, wz = (REAL)1 - wz2;                                \
                const REAL *b = img + xi + yi * sy + zi * sz;                                      \
                out[id] = b[0] * wx * wy * wz + b[sz] * wx * wy * wz2 + b[sy] * wx * wy2 * wz +    \
                          b[sy + sz] * wx * wy2 * wz2 + b[1] * wx2 * wy * wz +                     \
                          b[1 + sz] * wx2 * wy * wz2 + b[1 + sy] * wx2 * wy2 * wz +                \
                          b[1 + sy + sz] * wx2 * wy2 * wz2;                                        \
            }

void or_deform_f32(const float *img, const float *mx, const float *my, const float *mz,
                   int nx, int ny, int nz, float *out)
{
    DEFORM_BODY(float, floorf)
}

void or_deform_f64(const double *img, const double *mx, const double *my, const double *mz,
                   int nx, int ny, int nz, double *out)
{
    DEFORM_BODY(double, floor)
}

/* ---- displacement-field inversion, nefct/cc/deform/deform_tex.cu.cc:78-99 ----
 * Fixed-point passes x <- -mx(p + d), y <- -my(p + d), z <- -mz(p + d) from
 * d = 0, trilinear sampling with clamp-to-edge addressing (the reference
 * samples a clamp-addressed linear-filtered texture at texel centres). */
static float clamp_lerp3_f32(const float *m, float px, float py, float pz, int nx, int ny, int nz)
{
    const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
    const float ax = px - fx, ay = py - fy, az = pz - fz;
#define CL(v, n) ((v) < 0 ? 0 : ((v) > (n) - 1 ? (n) - 1 : (v)))
    const int x0 = CL((int)fx, nx), x1 = CL((int)fx + 1, nx);
    const int y0 = CL((int)fy, ny), y1 = CL((int)fy + 1, ny);
    const int z0 = CL((int)fz, nz), z1 = CL((int)fz + 1, nz);
#undef CL
    const long long sy = nx, sz = (long long)nx * ny;
    const float c00 = m[x0 + y0 * sy + z0 * sz] * (1.f - ax) + m[x1 + y0 * sy + z0 * sz] * ax;
    const float c10 = m[x0 + y1 * sy + z0 * sz] * (1.f - ax) + m[x1 + y1 * sy + z0 * sz] * ax;
    const float c01 = m[x0 + y0 * sy + z1 * sz] * (1.f - ax) + m[x1 + y0 * sy + z1 * sz] * ax;
    const float c11 = m[x0 + y1 * sy + z1 * sz] * (1.f - ax) + m[x1 + y1 * sy + z1 * sz] * ax;
    const float c0 = c00 * (1.f - ay) + c10 * ay, c1 = c01 * (1.f - ay) + c11 * ay;
    return c0 * (1.f - az) + c1 * az;
}

void or_warp_invert_f32(const float *mx, const float *my, const float *mz, int nx, int ny, int nz, int iters,
                        float *ix, float *iy, float *iz)
{
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                float u = 0.f, v = 0.f, w = 0.f;
                for (int it = 0; it < iters; ++it) {
                    u = -clamp_lerp3_f32(mx, x + u, y + v, z + w, nx, ny, nz);
                    v = -clamp_lerp3_f32(my, x + u, y + v, z + w, nx, ny, nz);
                    w = -clamp_lerp3_f32(mz, x + u, y + v, z + w, nx, ny, nz);
                }
                const long long id = x + (long long)y * nx + (long long)z * nx * ny;
                ix[id] = u; iy[id] = v; iz[id] = w;
            }
}

/* ---- distance-driven FDK backprojection, nefct/cc/distance_3d/dist_3d_back_fdk.cu.cc:17-255 ----
 * Detector-driven: every detector bin (ia, ib, iv) walks the slabs of its
 * driving axis (x when |x21| > |y21|, else y); in each slab its transverse
 * footprint is the span of the four rays through the bin's left/right edges
 * (edge x and y components paired both ways, :100-123, :200-223) and its z
 * footprint the span of the bin's lower/upper z edges (:125-139); every
 * overlapped voxel receives value * (overlap fraction in each axis) / |x21|
 * (or |y21|) * |p2 - p1| * SAD^2 / (SAD + x cos + y sin)^2 (:148-154).
 * Voxel units, grid centred on the axis, SID = source-detector and SAD =
 * source-axis (the python naming used there).  The float/double promotions
 * of the reference expressions are spelled out.  The (view, row) pairs form
 * OR_CHUNKS fixed chunks with private volumes summed in chunk order, as in
 * the reference build's shim, so the two agree bit for bit. */
#define DD_ABS(x) (((x) > 0) ? (x) : -(x))
#define DD_MIN(a, b) (((a) < (b)) ? (a) : (b))
#define DD_MAX(a, b) (((a) > (b)) ? (a) : (b))

static float dd_center(int i, float d, float o, int n)       /* (i + 0.5) * d + o - n * d / 2 */
{
    return (float)(((double)i + 0.5) * (double)d + (double)o - (double)((float)n * d / 2.0f));
}

static float dd_edge(int i, float d, float o, int n)         /* i * d + o - n * d / 2 (float) */
{
    return (float)i * d + o - (float)n * d / 2.0f;
}

static void dd_bin(int cyl, const float *cs, const float *sn, const float *off, float SID, float SAD, int nx,
                   int ny, int nz, float da, float ai, int na, float db, float bi, int nb, int ia, int ib, int iv,
                   int use_cosf, float value, float *img)
{
    const float cphi = cs[iv], sphi = sn[iv];
    const float x1 = -SAD * cphi, y1 = -SAD * sphi, z1 = off[iv];
    float x20, y20;
    if (!cyl) {
        x20 = SID - SAD;
        y20 = dd_center(ia, da, ai, na);
    } else {
        const float ang = dd_center(ia, da, ai, na);
        const float ca = use_cosf ? cosf(ang) : (float)cos((double)ang);
        const float sa = use_cosf ? sinf(ang) : (float)sin((double)ang);
        x20 = SID * ca - SAD;
        y20 = SID * sa;
    }
    const float z20 = dd_center(ib, db, bi, nb);
    const float x2 = x20 * cphi - y20 * sphi, y2 = x20 * sphi + y20 * cphi, z2 = z20 + off[iv];
    const float x21 = x2 - x1, y21 = y2 - y1, z21 = z2 - z1;
    /* the bin's left / right edge directions (the reference recomputes them per slab) */
    float e[2][2];
    for (int s = 0; s < 2; ++s) {
        float ex, ey;
        if (!cyl) {
            ex = SID - SAD;
            ey = dd_edge(ia + s, da, ai, na);
        } else {
            const float ang = dd_edge(ia + s, da, ai, na);
            const float ca = use_cosf ? cosf(ang) : (float)cos((double)ang);
            const float sa = use_cosf ? sinf(ang) : (float)sin((double)ang);
            ex = SID * ca - SAD;
            ey = SID * sa;
        }
        e[s][0] = ex * cphi - ey * sphi - x1;
        e[s][1] = ex * sphi + ey * cphi - y1;
    }
    const float xl = e[0][0], yl = e[0][1], xr = e[1][0], yr = e[1][1];
    const float len = sqrtf(x21 * x21 + y21 * y21 + z21 * z21);
    const int xdrive = DD_ABS(x21) > DD_ABS(y21);
    /* u: driving axis, v: transverse axis */
    const int nu = xdrive ? nx : ny, nv_ = xdrive ? ny : nx;
    const float u1 = xdrive ? x1 : y1, v1 = xdrive ? y1 : x1, u21 = xdrive ? x21 : y21;
    /* transverse ratios in the reference's pairing: v_l/u_l, v_l/u_r, v_r/u_l, v_r/u_r */
    const float vl = xdrive ? yl : xl, vr = xdrive ? yr : xr, ul = xdrive ? xl : yl, ur = xdrive ? xr : yr;
    for (int iu = 0; iu < nu; ++iu) {
        const float uc = (float)iu + 0.5f - (float)nu / 2 - u1;
        const float c0 = vl / ul * uc + v1 + (float)(nv_ / 2);
        const float c1 = vl / ur * uc + v1 + (float)(nv_ / 2);
        const float c2 = vr / ul * uc + v1 + (float)(nv_ / 2);
        const float c3 = vr / ur * uc + v1 + (float)(nv_ / 2);
        const float vi1 = DD_MIN(DD_MIN(c0, c1), DD_MIN(c2, c3));
        const float vi2 = DD_MAX(DD_MAX(c0, c1), DD_MAX(c2, c3));
        const int Vi1 = (int)floorf(vi1), Vi2 = (int)floorf(vi2);
        const float zl = z21 - db / 2, zr = z21 + db / 2;
        const float czl = zl / u21 * uc + z1 + (float)(nz / 2);
        const float czr = zr / u21 * uc + z1 + (float)(nz / 2);
        const float zi1 = DD_MIN(czl, czr), zi2 = DD_MAX(czl, czr);
        const int Zi1 = (int)floorf(zi1), Zi2 = (int)floorf(zi2);
        for (int iv2 = DD_MAX(0, Vi1); iv2 <= DD_MIN(nv_ - 1, Vi2); ++iv2) {
            float wv = DD_MIN(iv2 + 1.0f, vi2) - DD_MAX(iv2 + 0.0f, vi1);
            wv /= (vi2 - vi1);
            for (int iz = DD_MAX(0, Zi1); iz <= DD_MIN(nz - 1, Zi2); ++iz) {
                float wz = DD_MIN(iz + 1.0f, zi2) - DD_MAX(iz + 0.0f, zi1);
                wz /= (zi2 - zi1);
                const int ix = xdrive ? iu : iv2, iy = xdrive ? iv2 : iu;
                const float xc = (float)(ix + 0.5 - nx / 2), yc = (float)(iy + 0.5 - ny / 2);
                float weight = wv * wz / DD_ABS(u21) * len;
                weight *= SAD * SAD / (SAD + xc * cphi + yc * sphi) / (SAD + xc * cphi + yc * sphi);
                img[ix + (long long)iy * nx + (long long)iz * nx * ny] += value * weight;
            }
        }
    }
}

void or_dd_backproject_f32(const float *proj, const float *cs, const float *sn, const float *off, int nv,
                           float SID, float SAD, int nx, int ny, int nz, int na, float da, float ai, int nb,
                           float db, float bi, int cyl, int use_cosf, float *img)
{
    const long long nvox = (long long)nx * ny * nz, rows = (long long)nv * nb;
    float *priv = (float *)calloc((size_t)OR_CHUNKS * nvox, sizeof(float));
    #pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < OR_CHUNKS; ++c) {
        float *mine = priv + (long long)c * nvox;
        for (long long r = rows * c / OR_CHUNKS; r < rows * (c + 1) / OR_CHUNKS; ++r) {
            const int iv = (int)(r / nb), ib = (int)(r % nb);
            for (int ia = 0; ia < na; ++ia)
                dd_bin(cyl, cs, sn, off, SID, SAD, nx, ny, nz, da, ai, na, db, bi, nb, ia, ib, iv, use_cosf,
                       proj[ia + (long long)ib * na + (long long)iv * na * nb], mine);
        }
    }
    #pragma omp parallel for schedule(static)
    for (long long i = 0; i < nvox; ++i) {
        float s = 0.0f;
        for (int c = 0; c < OR_CHUNKS; ++c) s += priv[(long long)c * nvox + i];
        img[i] = s;
    }
    free(priv);
}
#undef DD_ABS
#undef DD_MIN
#undef DD_MAX
