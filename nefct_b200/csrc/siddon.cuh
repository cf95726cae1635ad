// Slab-split ray walk on sm_100a.
//
// Semantics follow the reference's per-ray routine project_device /
// backproject_device (nefct/cc/siddon_3d/siddon.cu.cc:12-321, 450-764;
// cpp/siddon/siddon_gpu.cu.cc:11-650): normalise the ray to x-pitch voxel
// units, drive along x when |xd| >= |yd| (or > with NEFCT_TIE_GT), and
// split each driving slab's length among at most three voxels from the
// transverse crossing ratios, pairing (v1, w1) first (quirk Q1).
//
// GPU structure (not the reference's):
//  * every position that feeds a floor() or a comparison is evaluated with
//    explicit round-to-nearest operations in the reference's order, so the
//    voxel choices are identical to the reference's; each plane position is
//    computed once and carried to the next slab;
//  * the per-contribution weight is r * W with W = S*dx/L^2 hoisted per ray
//    (the reference re-evaluates r*S*dx/L/L per contribution; the results
//    differ by rounding only);
//  * the slab range is clipped in FP64 to the slabs where the ray can touch
//    the volume (with a one-voxel margin); slabs outside contribute nothing,
//    so the clip changes no result, only the trip count;
//  * the three-way case split is written as one predicated sequence of at
//    most three (voxel, weight) slots, in the reference's accumulation order.
#pragma once

#include "common.cuh"

namespace nefct {

template <typename T> struct GridDev {
    int nx, ny, nz;
    T cx, cy, cz;
    T dx_, dy, dz;      // dx_ = sx/nx, dy = sy/ny/dx_, dz = sz/nz/dx_ (reference :19-22)
    T nx2, ny2, nz2;    // n/2.0f (:34-36)
};

// Host-side construction with the reference's float operations.
template <typename T> inline GridDev<T> make_grid_dev(const nefct_grid &g)
{
    GridDev<T> d;
    d.nx = g.nx; d.ny = g.ny; d.nz = g.nz;
    d.cx = (T)g.cx; d.cy = (T)g.cy; d.cz = (T)g.cz;
    d.dx_ = (T)g.sx / (T)g.nx;
    d.dy = (T)g.sy / (T)g.ny / d.dx_;
    d.dz = (T)g.sz / (T)g.nz / d.dx_;
    d.nx2 = (T)g.nx / (T)2; d.ny2 = (T)g.ny / (T)2; d.nz2 = (T)g.nz / (T)2;
    return d;
}

template <typename T> struct Walk {
    T pu, pv, pw;        // source in voxel units along (drive, other transverse, z)
    T kv, kw;            // slopes d(v)/d(u), d(z)/d(u)
    T dv, nu2, nv2;
    T W, Wmid;           // contribution weights (Wmid: three-voxel middle slot, Q5)
    int nu, nv, k0, k1;  // slab count, transverse extent, inclusive slab range
    bool xdrive, vdiv;
};

// Clips the slab range of the driving axis to [k0, k1] (FP64): slab k lies
// between planes t = k - nu2 and t + 1; position p(t) = A + B t must reach
// [-1, n + 1] for the slab to be able to touch the volume.
__device__ __forceinline__ void clip_axis(double A, double B, int n, double nu2, int nu, int &k0, int &k1)
{
    const double lo = -1.0, hi = (double)n + 1.0;
    if (B == 0.0) {
        if (A < lo || A > hi) { k0 = 1; k1 = 0; }
        return;
    }
    double t0 = (lo - A) / B, t1 = (hi - A) / B;
    if (t0 > t1) { const double s = t0; t0 = t1; t1 = s; }
    // k >= t0 + nu2 - 1 and k <= t1 + nu2; clamp before converting
    double a = ceil(t0 + nu2 - 1.0), b = floor(t1 + nu2);
    a = fmin(fmax(a, -1.0), (double)nu + 1.0);
    b = fmax(fmin(b, (double)nu), -2.0);
    k0 = max(k0, (int)a);
    k1 = min(k1, (int)b);
}

// Per-ray setup of project_device / backproject_device (reference :19-44,
// :181-184; :457-483).  Returns false when the ray contributes nothing.
template <typename T>
__device__ __forceinline__ bool setup_walk(const GridDev<T> &g, const T *r, uint32_t flags, Walk<T> &w)
{
    using F = FP<T>;
    const T x1 = F::div(F::sub(r[0], g.cx), g.dx_), x2 = F::div(F::sub(r[3], g.cx), g.dx_);
    const T y1 = F::div(F::sub(r[1], g.cy), g.dx_), y2 = F::div(F::sub(r[4], g.cy), g.dx_);
    const T z1 = F::div(F::sub(r[2], g.cz), g.dx_), z2 = F::div(F::sub(r[5], g.cz), g.dx_);
    const T xd = F::sub(x2, x1), yd = F::sub(y2, y1), zd = F::sub(z2, z1);
    const T xy2 = F::add(F::mul(xd, xd), F::mul(yd, yd));
    if ((flags & NEFCT_SKIP_SHORT) && F::sqrt(xy2) < (T)10) return false;   // Q4
    // a ray along z has 0/0 slopes in the reference (undefined); it contributes 0 here
    if (xy2 == (T)0) return false;
    const T L = F::sqrt(F::add(xy2, F::mul(zd, zd)));
    const T axd = xd > (T)0 ? xd : -xd, ayd = yd > (T)0 ? yd : -yd;
    w.xdrive = (flags & NEFCT_TIE_GT) ? (axd > ayd) : (axd >= ayd);
    if (w.xdrive) {
        w.nu = g.nx; w.nv = g.ny; w.pu = x1; w.pv = y1;
        w.kv = F::div(yd, xd); w.kw = F::div(zd, xd);
        w.dv = g.dy; w.vdiv = g.dy != (T)1; w.nu2 = g.nx2; w.nv2 = g.ny2;
    } else {
        // the y-driven branch of the reference has no division by the x pitch (:194-200)
        w.nu = g.ny; w.nv = g.nx; w.pu = y1; w.pv = x1;
        w.kv = F::div(xd, yd); w.kw = F::div(zd, yd);
        w.dv = (T)1; w.vdiv = false; w.nu2 = g.ny2; w.nv2 = g.nx2;
    }
    w.pw = z1;
    const T S = F::sqrt(F::add(F::add((T)1, F::mul(w.kv, w.kv)), F::mul(w.kw, w.kw)));
    T W = F::mul(S, g.dx_);
    if (!(flags & NEFCT_NO_INV_L2)) W = F::div(F::div(W, L), L);
    w.W = W;
    w.Wmid = ((flags & NEFCT_Q5) && !w.xdrive) ? F::div(W, L) : W;

    w.k0 = 0; w.k1 = w.nu - 1;
    const double pu = (double)w.pu, kv = (double)w.kv, kw = (double)w.kw;
    const double dv = (double)w.dv, dz = (double)g.dz;
    clip_axis(((double)w.pv - kv * pu) / dv + (double)w.nv2, kv / dv, w.nv, (double)w.nu2, w.nu, w.k0, w.k1);
    clip_axis(((double)w.pw - kw * pu) / dz + (double)g.nz2, kw / dz, g.nz, (double)w.nu2, w.nu, w.k0, w.k1);
    w.k0 = max(w.k0, 0);
    w.k1 = min(w.k1, w.nu - 1);
    return w.k0 <= w.k1;
}

// Visits every (slab, v, z, ratio, weight) contribution of the ray in the
// reference's order.  op(k, cv, cw, r, Wslot) is called for admitted voxels.
template <typename T, class Op>
__device__ __forceinline__ void run_walk(const Walk<T> &w, const GridDev<T> &g, Op &op)
{
    using F = FP<T>;
    const bool sv = w.kv >= (T)0, sw = w.kw >= (T)0;
    const bool zdiv = g.dz != (T)1;
    const int nv = w.nv, nz = g.nz;
    auto posv = [&](T t) {
        T q = F::add(w.pv, F::mul(w.kv, F::sub(t, w.pu)));
        if (w.vdiv) q = F::div(q, w.dv);
        return F::add(q, w.nv2);
    };
    auto posw = [&](T t) {
        T q = F::add(w.pw, F::mul(w.kw, F::sub(t, w.pu)));
        if (zdiv) q = F::div(q, g.dz);
        return F::add(q, g.nz2);
    };
    T t = F::sub((T)w.k0, w.nu2);
    T qav = posv(t), qaw = posw(t);
    int fav = F::ifloor(qav), faw = F::ifloor(qaw);
    for (int k = w.k0; k <= w.k1; ++k) {
        const T t2 = F::add(t, (T)1);
        const T qbv = posv(t2), qbw = posw(t2);
        const int fbv = F::ifloor(qbv), fbw = F::ifloor(qbw);
        const T q1v = sv ? qav : qbv, q2v = sv ? qbv : qav;
        const T q1w = sw ? qaw : qbw, q2w = sw ? qbw : qaw;
        const int cv1 = sv ? fav : fbv, cv2 = sv ? fbv : fav;
        const int cw1 = sw ? faw : fbw, cw2 = sw ? fbw : faw;
        t = t2; qav = qbv; qaw = qbw; fav = fbv; faw = fbw;

        const bool vx = cv1 != cv2, wx = cw1 != cw2;
        // slab admission (reference :80, :92, :112, :116, :132)
        if (cv1 >= nv || cv1 < (vx ? -1 : 0) || cw1 >= nz || cw1 < (wx ? -1 : 0)) continue;
        T rv = (T)1, rw = (T)1;
        if (vx) rv = F::div(F::sub((T)cv2, q1v), F::sub(q2v, q1v));
        if (wx) rw = F::div(F::sub((T)cw2, q1w), F::sub(q2w, q1w));
        const bool vfirst = rv > rw;   // middle voxel (cv1, cw2) when true, else (cv2, cw1)
        if (cv1 >= 0 && cw1 >= 0) op(k, cv1, cw1, vfirst ? rw : rv, w.W);
        if (vx || wx) {
            const int mv = vfirst ? cv1 : cv2, mw = vfirst ? cw2 : cw1;
            const T rm = vfirst ? F::sub(rv, rw) : F::sub(rw, rv);
            if ((unsigned)mv < (unsigned)nv && (unsigned)mw < (unsigned)nz)
                op(k, mv, mw, rm, (vx && wx) ? w.Wmid : w.W);
            if (vx && wx && cv2 < nv && cw2 < nz)
                op(k, cv2, cw2, F::sub((T)1, vfirst ? rv : rw), w.W);
        }
    }
}

}  // namespace nefct
