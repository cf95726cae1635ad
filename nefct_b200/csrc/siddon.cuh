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
//    most three (voxel, weight) slots, in the reference's accumulation order;
//  * the crossing ratios use the approximate reciprocal (<= 2 ulp) in FP32:
//    they only scale weights, and the split is continuous in them;
//  * the per-ray weight W is applied once to the ray's sum of value * ratio
//    (rounding-level difference from the per-contribution products);
//  * slabs whose candidate voxels are all inside the grid skip the range
//    checks (interior range computed with the clip).
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

// Scanner constants of the cone-beam ray generator.
template <typename T> struct RayGeom {
    T src_iso, src_det, da, ai, db, bi, half_a, half_b;
    int cyl;
};

template <typename T> inline RayGeom<T> make_ray_geom(const nefct_cb_geom &g)
{
    RayGeom<T> r;
    r.src_iso = (T)g.src_iso; r.src_det = (T)g.src_det;
    r.da = (T)g.da; r.ai = (T)g.a_shift; r.db = (T)g.db; r.bi = (T)g.b_shift;
    // na*da/2 in the reference's order (siddon.cu.cc:341)
    r.half_a = (T)g.na * r.da / (T)2;
    r.half_b = (T)g.nb * r.db / (T)2;
    r.cyl = g.det_kind == NEFCT_DET_CYL;
    return r;
}

// Ray of detector cell (ia, ib) at a view with (cos, sin, z offset) =
// (cs, sn, off): ProjectFlatKernel (siddon.cu.cc:341-353) /
// ProjectCyliKernel (:376-387), same order of operations, plus the optional
// z offset of source and detector.  r = (x1, y1, z1, x2, y2, z2).
template <typename T>
__device__ __forceinline__ void cb_ray(const RayGeom<T> &p, T cs, T sn, T off, int ia, int ib, T *r)
{
    using F = FP<T>;
    const T a = F::sub(F::mul(F::add(p.ai, (T)ia), p.da), p.half_a);
    const T b = F::sub(F::mul(F::add(p.bi, (T)ib), p.db), p.half_b);
    T xd0, yd0;
    if (p.cyl) {
        xd0 = F::sub(F::mul(p.src_det, cos(a)), p.src_iso);
        yd0 = F::mul(p.src_det, sin(a));
    } else {
        xd0 = F::sub(p.src_det, p.src_iso);
        yd0 = a;
    }
    r[0] = F::mul(-p.src_iso, cs);
    r[1] = F::mul(-p.src_iso, sn);
    r[2] = F::add((T)0, off);
    r[3] = F::sub(F::mul(xd0, cs), F::mul(yd0, sn));
    r[4] = F::add(F::mul(xd0, sn), F::mul(yd0, cs));
    r[5] = F::add(b, off);
}

template <typename T> struct Walk {
    T pu, pv, pw;        // source in voxel units along (drive, other transverse, z)
    T kv, kw;            // slopes d(v)/d(u), d(z)/d(u)
    T dv, nu2, nv2;
    T W, Wmid;           // contribution weights (Wmid: three-voxel middle slot, Q5)
    int nu, nv, k0, k1;  // slab count, transverse extent, inclusive slab range
    int ki0, ki1;        // interior slabs: every candidate voxel is inside the grid
    bool xdrive, vdiv;
};

// Slab ranges of the driving axis (FP64).  Slab k lies between planes
// t = k - nu2 and t + 1, and the transverse position is p(t) = A + B t.
// [k0, k1]: slabs whose positions reach [-1 - m, n + 1 + m], i.e. that can
// touch the grid.  [ki0, ki1]: slabs whose positions at both planes lie in
// [m, n - m], so the floors of both planes are valid indices and no range
// check is needed.  m covers the difference between these FP64 positions and
// the FP32 ones the walk evaluates: 1/64 voxel plus 1e-5 of the largest
// magnitude entering them (a few hundred FP32 ulps).
__device__ __forceinline__ void clip_axis(double A, double B, int n, double nu2, int nu, double mag, int &k0,
                                          int &k1, int &ki0, int &ki1)
{
    const double m = 1.0 / 64.0 + 1e-5 * mag;
    if (B == 0.0) {
        if (A < -1.0 - m || A > (double)n + 1.0 + m) { k0 = 1; k1 = 0; }
        if (A < m || A > (double)n - m) { ki0 = 1; ki1 = 0; }
        return;
    }
    auto span = [&](double lo, double hi, double &t0, double &t1) {
        t0 = (lo - A) / B;
        t1 = (hi - A) / B;
        if (t0 > t1) { const double s = t0; t0 = t1; t1 = s; }
    };
    auto clampk = [&](double v) { return (int)fmin(fmax(v, -2.0), (double)nu + 1.0); };
    double t0, t1;
    span(-1.0 - m, (double)n + 1.0 + m, t0, t1);
    k0 = max(k0, clampk(ceil(t0 + nu2 - 1.0)));
    k1 = min(k1, clampk(floor(t1 + nu2)));
    span(m, (double)n - m, t0, t1);
    ki0 = max(ki0, clampk(ceil(t0 + nu2)));
    ki1 = min(ki1, clampk(floor(t1 + nu2) - 1.0));
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
    w.ki0 = 0; w.ki1 = w.nu - 1;
    const double pu = (double)w.pu, kv = (double)w.kv, kw = (double)w.kw;
    const double dv = (double)w.dv, dz = (double)g.dz;
    const double mag = fabs(pu) + fabs((double)w.pv) + fabs((double)w.pw) + (double)(w.nu + w.nv + g.nz);
    clip_axis(((double)w.pv - kv * pu) / dv + (double)w.nv2, kv / dv, w.nv, (double)w.nu2, w.nu, mag, w.k0, w.k1,
              w.ki0, w.ki1);
    clip_axis(((double)w.pw - kw * pu) / dz + (double)g.nz2, kw / dz, g.nz, (double)w.nu2, w.nu, mag, w.k0, w.k1,
              w.ki0, w.ki1);
    w.k0 = max(w.k0, 0);
    w.k1 = min(w.k1, w.nu - 1);
    w.ki0 = max(w.ki0, w.k0);
    w.ki1 = min(w.ki1, w.k1);
    return w.k0 <= w.k1;
}

// Floors of plane positions.  FP32: floor(q) + 1.5*2^23 equals
// round-down(q + 1.5*2^23) exactly for |q| < 2^22 (the sum lies in
// [2^23, 2^24), where the float spacing is 1); the float floor is that sum
// minus 1.5*2^23 (exact) and the integer floor its bit pattern minus
// 0x4B400000, so no conversion instruction is needed.  Interior slabs have
// positions inside the grid; boundary slabs clamp the positions to +-2^21
// first (grid dimensions are limited to 2^20, so a clamped position stays
// outside the grid and its voxels stay rejected).  FP64 converts.
constexpr float kFloorMagic = 12582912.0f;   // 1.5 * 2^23
constexpr int kFloorMagicBits = 0x4B400000;
constexpr float kFloorClamp = 2097152.0f;    // 2^21

template <bool CHECK> __device__ __forceinline__ float magic_floor(float q)
{
    if (CHECK) q = fminf(fmaxf(q, -kFloorClamp), kFloorClamp);
    return __fadd_rd(q, kFloorMagic);
}

template <bool CHECK> __device__ __forceinline__ float2 magic_floor2(float2 q)
{
    if (CHECK) q = make_float2(fminf(fmaxf(q.x, -kFloorClamp), kFloorClamp), fminf(fmaxf(q.y, -kFloorClamp), kFloorClamp));
    return __fadd2_rd(q, make_float2(kFloorMagic, kFloorMagic));
}

// Floor records M of a position: FP32 the biased float above, FP64 the int.
//   value2(a, b)  the two floors as T;  biased(m)  floor + bias as unsigned;
//   to_int(m)     the floor.
template <typename T> struct Floor;
template <> struct Floor<float> {
    using M = float;
    static constexpr unsigned kBias = (unsigned)kFloorMagicBits;
    template <bool CHECK> static __device__ __forceinline__ void of2(Pair<float> q, M &a, M &b)
    {
        const float2 m = magic_floor2<CHECK>(q.v);
        a = m.x; b = m.y;
    }
    static __device__ __forceinline__ Pair<float> value2(M a, M b)
    {
        Pair<float> p;
        p.v = __fadd2_rn(make_float2(a, b), make_float2(-kFloorMagic, -kFloorMagic));
        return p;
    }
    static __device__ __forceinline__ unsigned biased(M m) { return (unsigned)__float_as_int(m); }
    static __device__ __forceinline__ int to_int(M m) { return __float_as_int(m) - kFloorMagicBits; }
};
template <> struct Floor<double> {
    using M = int;
    static constexpr unsigned kBias = 0u;
    template <bool CHECK> static __device__ __forceinline__ void of2(Pair<double> q, M &a, M &b)
    {
        a = __double2int_rd(q.x());
        b = __double2int_rd(q.y());
    }
    static __device__ __forceinline__ Pair<double> value2(M a, M b) { return Pair<double>::make((double)a, (double)b); }
    static __device__ __forceinline__ unsigned biased(M m) { return (unsigned)m; }
    static __device__ __forceinline__ int to_int(M m) { return m; }
};

// The up-to-three contributions of one driving slab: flat volume index,
// split ratio r (the weight is r * W) and activity, in the reference's order.
template <typename T> struct SlabSlots {
    unsigned idx[3];
    T r[3];
    bool ok[3];
    bool mid3;          // slot 1 is the middle entry of a three-voxel split (Q5)
};

// Walks the slabs of one ray, carrying the plane positions, their floors and
// the z row offsets from one slab to the next.
//   DIV   the grid is not cubic: positions divide by dy (x-driven) / dz;
//   SWP   the z slope is >= 0 (uniform along a detector row, so along a warp);
//   VUP   the transverse slope kv is >= 0, so the v position grows along the
//         walk (the entry plane is the low one; rounding is monotone, so this
//         equals the reference's min/max choice);
//   SV1   the transverse stride is 1 (x-fastest volume for y-driven rays,
//         y-fastest copy for x-driven rays);
//   EXACT crossing ratios by exact division (the intersection count).
// next<CHECK>() returns the next slab's contributions; CHECK=false is only
// valid for interior slabs, where all candidate voxels are inside the grid.
// Indices are computed modulo 2^32 from biased floors; for admitted voxels
// the biases cancel and the index is exact.
template <typename T, bool DIV, bool SWP, bool VUP, bool SV1, bool EXACT = false> struct Walker {
    using F = FP<T>;
    using P2 = Pair<T>;
    using FL = Floor<T>;
    using M = typename FL::M;
    P2 p0, k2, n2;          // (pv, pw), (kv, kw), (nv2, nz2)
    T pu, dv, dz;
    int nv, nz, su, sv, sw;
    unsigned base;          // k * su minus the floors' biases
    bool vdiv, zdiv;
    T t, qav, qaw;
    M mav, maw;
    unsigned rowa;

    // Positions of plane t in v and z: ((p + k * (t - pu)) [/ d]) + n/2, the
    // reference's order (:54-55, :67-68, :194-195, :207-208), both axes at once.
    __device__ __forceinline__ P2 pos(T tt) const
    {
        const T d = F::sub(tt, pu);
        P2 q = P2::add(p0, P2::mul(k2, P2::make(d, d)));
        if (DIV && (vdiv || zdiv))
            q = P2::make(vdiv ? F::div(q.x(), dv) : q.x(), zdiv ? F::div(q.y(), dz) : q.y());
        return P2::add(q, n2);
    }

    __device__ __forceinline__ Walker(const Walk<T> &w, const GridDev<T> &g, int k, int su_, int sv_, int sw_)
    {
        p0 = P2::make(w.pv, w.pw);
        k2 = P2::make(w.kv, w.kw);
        n2 = P2::make(w.nv2, g.nz2);
        pu = w.pu; dv = w.dv; dz = g.dz;
        nv = w.nv; nz = g.nz; su = su_; sv = SV1 ? 1 : sv_; sw = sw_;
        vdiv = w.vdiv;
        zdiv = dz != (T)1;
        base = (unsigned)k * (unsigned)su - FL::kBias * ((unsigned)sv + (unsigned)sw);
        t = F::sub((T)k, w.nu2);
        const P2 q = pos(t);
        qav = q.x();
        qaw = q.y();
        FL::template of2<true>(q, mav, maw);
        rowa = FL::biased(maw) * (unsigned)sw;
    }

    template <bool CHECK> __device__ __forceinline__ SlabSlots<T> next()
    {
        const T t2 = F::add(t, (T)1);
        const P2 qb = pos(t2);
        const T qbv = qb.x(), qbw = qb.y();
        M mbv, mbw;
        FL::template of2<CHECK>(qb, mbv, mbw);
        const unsigned rowb = FL::biased(mbw) * (unsigned)sw;
        // low/high plane of the slab in v and z (static by the slope signs)
        const T q1v = VUP ? qav : qbv, q2v = VUP ? qbv : qav;
        const M m1v = VUP ? mav : mbv, m2v = VUP ? mbv : mav;
        const T q1w = SWP ? qaw : qbw, q2w = SWP ? qbw : qaw;
        const M m1w = SWP ? maw : mbw, m2w = SWP ? mbw : maw;
        const unsigned row1 = SWP ? rowa : rowb, row2 = SWP ? rowb : rowa;
        const unsigned b = base;
        t = t2; qav = qbv; qaw = qbw; mav = mbv; maw = mbw; rowa = rowb; base += (unsigned)su;

        const bool vx = m1v != m2v, wx = m1w != m2w;
        // crossing ratios (c2 - q1) / (q2 - q1) of both axes (reference :94, :118, :134-135)
        const P2 nq1 = P2::make(-q1v, -q1w);
        const P2 num = P2::add(FL::value2(m2v, m2w), nq1);
        const P2 den = P2::add(P2::make(q2v, q2w), nq1);
        const T rvq = EXACT ? F::div(num.x(), den.x()) : F::ratio(num.x(), den.x());
        const T rwq = EXACT ? F::div(num.y(), den.y()) : F::ratio(num.y(), den.y());
        const T rv = vx ? rvq : (T)1, rw = wx ? rwq : (T)1;
        const bool vfirst = rv > rw;   // middle voxel (cv1, cw2) when true, else (cv2, cw1)
        const unsigned V1 = FL::biased(m1v) * (unsigned)sv, V2 = FL::biased(m2v) * (unsigned)sv;
        SlabSlots<T> s;
        s.r[0] = F::min(rv, rw);
        s.r[1] = F::abs(F::sub(rv, rw));
        s.r[2] = F::sub((T)1, F::max(rv, rw));
        s.idx[0] = b + V1 + row1;
        s.idx[1] = b + (vfirst ? V1 + row2 : V2 + row1);
        s.idx[2] = b + V2 + row2;
        s.mid3 = vx && wx;
        if (CHECK) {
            // slab admission (reference :80, :92, :112, :116, :132)
            const int cv1 = FL::to_int(m1v), cv2 = FL::to_int(m2v), cw1 = FL::to_int(m1w), cw2 = FL::to_int(m2w);
            const bool adm = (unsigned)(cv1 + (int)vx) < (unsigned)(nv + (int)vx) &&
                             (unsigned)(cw1 + (int)wx) < (unsigned)(nz + (int)wx);
            const int mv = vfirst ? cv1 : cv2, mw = vfirst ? cw2 : cw1;
            s.ok[0] = adm && (cv1 | cw1) >= 0;
            s.ok[1] = adm && (vx || wx) && (unsigned)mv < (unsigned)nv && (unsigned)mw < (unsigned)nz;
            s.ok[2] = adm && vx && wx && cv2 < nv && cw2 < nz;
        } else {
            s.ok[0] = true;
            s.ok[1] = vx || wx;
            s.ok[2] = vx && wx;
        }
        return s;
    }
};

// Runs f(slots) over slabs [a, b] with the given check mode (unrolled by two
// so the carried plane state alternates registers instead of being moved).
template <bool CHECK, class WK, class Fn>
__device__ __forceinline__ void walk_range(WK &it, int a, int b, Fn &f)
{
#pragma unroll 2
    for (int k = a; k <= b; ++k) f(it.template next<CHECK>());
}

// Visits the slabs k0..k1 of a ray: boundary slabs with range checks,
// interior slabs without.
template <class WK, class Fn>
__device__ __forceinline__ void walk_all(WK &it, const int k0, const int k1, const int ki0, const int ki1, Fn &f)
{
    if (ki0 <= ki1) {
        walk_range<true>(it, k0, ki0 - 1, f);
        walk_range<false>(it, ki0, ki1, f);
        walk_range<true>(it, ki1 + 1, k1, f);
    } else {
        walk_range<true>(it, k0, k1, f);
    }
}

// Calls body(Walker<...>) with the walker variant of the ray's slope signs.
template <typename T, bool DIV, bool SV1, bool EXACT = false, class Body>
__device__ __forceinline__ void with_walker(const Walk<T> &w, const GridDev<T> &g, int su, int sv, int sw, Body &&body)
{
    if (w.kw >= (T)0) {
        if (w.kv >= (T)0) { Walker<T, DIV, true, true, SV1, EXACT> it(w, g, w.k0, su, sv, sw); body(it); }
        else { Walker<T, DIV, true, false, SV1, EXACT> it(w, g, w.k0, su, sv, sw); body(it); }
    } else {
        if (w.kv >= (T)0) { Walker<T, DIV, false, true, SV1, EXACT> it(w, g, w.k0, su, sv, sw); body(it); }
        else { Walker<T, DIV, false, false, SV1, EXACT> it(w, g, w.k0, su, sv, sw); body(it); }
    }
}

// Weighted sum of the volume along the ray (forward):
//   sum over contributions of v * r, times W (and Wmid for Q5 middles).
template <typename T, bool DIV, bool SV1, bool Q5>
__device__ __forceinline__ T gather_walk(const Walk<T> &w, const GridDev<T> &g, const T *__restrict__ base, int su,
                                         int sv, int sw)
{
    T acc = (T)0, accm = (T)0;
    auto f = [&](const SlabSlots<T> &s) {
        const T v0 = s.ok[0] ? __ldg(base + s.idx[0]) : (T)0;
        const T v1 = s.ok[1] ? __ldg(base + s.idx[1]) : (T)0;
        const T v2 = s.ok[2] ? __ldg(base + s.idx[2]) : (T)0;
        acc += v0 * s.r[0];
        if (Q5 && s.mid3) accm += v1 * s.r[1];
        else acc += v1 * s.r[1];
        acc += v2 * s.r[2];
    };
    with_walker<T, DIV, SV1>(w, g, su, sv, sw, [&](auto &it) { walk_all(it, w.k0, w.k1, w.ki0, w.ki1, f); });
    return Q5 ? acc * w.W + accm * w.Wmid : acc * w.W;
}

// Scatters value * weight along the ray (transpose); reductions do not wait
// for their result.
template <typename T, bool DIV, bool SV1, bool Q5>
__device__ __forceinline__ void scatter_walk(const Walk<T> &w, const GridDev<T> &g, T *base, int su, int sv, int sw,
                                             T value)
{
    const T yw = value * w.W, ym = value * w.Wmid;
    auto f = [&](const SlabSlots<T> &s) {
        if (s.ok[0]) atomicAdd(base + s.idx[0], yw * s.r[0]);
        if (s.ok[1]) atomicAdd(base + s.idx[1], ((Q5 && s.mid3) ? ym : yw) * s.r[1]);
        if (s.ok[2]) atomicAdd(base + s.idx[2], yw * s.r[2]);
    };
    with_walker<T, DIV, SV1>(w, g, su, sv, sw, [&](auto &it) { walk_all(it, w.k0, w.k1, w.ki0, w.ki1, f); });
}

// Deterministic transpose: each contribution value * weight is scaled by
// a power of two (exact) and rounded to a 64-bit integer; integer sums do
// not depend on the order of the reductions, so the result is bitwise
// reproducible.  The caller picks the scale so that no sum can overflow.
__device__ __forceinline__ long long to_fixed(float v) { return __float2ll_rn(v); }
__device__ __forceinline__ long long to_fixed(double v) { return __double2ll_rn(v); }

template <typename T, bool DIV, bool SV1>
__device__ __forceinline__ void scatter_walk_fixed(const Walk<T> &w, const GridDev<T> &g, unsigned long long *base,
                                                   int su, int sv, int sw, T value, T scale)
{
    const T yw = value * w.W;
    auto f = [&](const SlabSlots<T> &s) {
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (s.ok[j]) atomicAdd(base + s.idx[j], (unsigned long long)to_fixed((yw * s.r[j]) * scale));
    };
    with_walker<T, DIV, SV1>(w, g, su, sv, sw, [&](auto &it) { walk_all(it, w.k0, w.k1, w.ki0, w.ki1, f); });
}

// Number of contributions of the ray (the throughput unit).  Uses the
// reference's exact ratio division, so near-equal crossing ratios order the
// three-voxel split exactly as the reference does and the count matches it.
template <typename T, bool DIV>
__device__ __forceinline__ unsigned count_walk(const Walk<T> &w, const GridDev<T> &g)
{
    unsigned n = 0;
    auto f = [&](const SlabSlots<T> &s) { n += (unsigned)s.ok[0] + (unsigned)s.ok[1] + (unsigned)s.ok[2]; };
    with_walker<T, DIV, true, true>(w, g, 0, 1, 0, [&](auto &it) { walk_all(it, w.k0, w.k1, w.ki0, w.ki1, f); });
    return n;
}

// ---------------- exact Siddon (NEFCT_EXACT) ----------------
//
// Classical plane-crossing traversal (Siddon 1985; incremental form of
// Jacobs et al. 1998): the segment p1 -> p2 is clipped to the grid box and
// split at every x, y and z plane it crosses; each piece contributes its
// exact length times the voxel value.  FP64 is used only for the per-ray
// set-up -- entry/exit parameters alpha_min/alpha_max, the first voxel and
// the first plane crossings -- where FP32 cancellation would drop or
// duplicate pieces at grazing angles; the stepping runs in T (FP32 for the
// float build) from those values.  Weights: length (physical units) times
// 1/L^2 in x-pitch voxel units unless NEFCT_NO_INV_L2, as in the default
// walk.  The loop is bounded by nx + ny + nz + 4 steps.
template <typename T> struct ExactRay {
    T alpha, amax, ax, ay, az, dax, day, daz, scale;
    int i, j, k, di, dj, dk;
    bool xdom;                // |dx| >= |dy|: gather from the y-fastest copy
};

template <typename T>
__device__ __forceinline__ bool exact_setup(const GridDev<T> &g, const T *r, uint32_t flags, ExactRay<T> &e)
{
    const int n[3] = {g.nx, g.ny, g.nz};
    const double dx_ = (double)g.dx_;
    const double pitch[3] = {dx_, (double)g.dy * dx_, (double)g.dz * dx_};
    const double c[3] = {(double)g.cx, (double)g.cy, (double)g.cz};
    double p1[3], d[3], lo[3];
    double amin = 0.0, amax = 1.0;
    for (int a = 0; a < 3; ++a) {
        p1[a] = (double)r[a];
        d[a] = (double)r[a + 3] - p1[a];
        lo[a] = c[a] - 0.5 * n[a] * pitch[a];
        if (d[a] != 0.0) {
            double a0 = (lo[a] - p1[a]) / d[a], a1 = (lo[a] + n[a] * pitch[a] - p1[a]) / d[a];
            if (a0 > a1) { const double t = a0; a0 = a1; a1 = t; }
            amin = fmax(amin, a0);
            amax = fmin(amax, a1);
        } else if (p1[a] < lo[a] || p1[a] >= lo[a] + n[a] * pitch[a]) {
            return false;
        }
    }
    if (!(amax > amin)) return false;
    const double L = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if ((flags & NEFCT_SKIP_SHORT) && sqrt(d[0] * d[0] + d[1] * d[1]) / dx_ < 10.0) return false;
    int idx[3], step[3];
    double anext[3], dal[3];
    // first voxel: the one containing the middle of the first piece
    double first = amax;
    for (int a = 0; a < 3; ++a) {
        if (d[a] == 0.0) continue;
        const double s = (floor((p1[a] + amin * d[a] - lo[a]) / pitch[a]) + (d[a] > 0 ? 1.0 : 0.0)) * pitch[a] + lo[a];
        double ap = (s - p1[a]) / d[a];
        if (ap <= amin) ap += pitch[a] / fabs(d[a]);
        first = fmin(first, ap);
    }
    const double am = 0.5 * (amin + first);
    for (int a = 0; a < 3; ++a) {
        int i = (int)floor((p1[a] + am * d[a] - lo[a]) / pitch[a]);
        i = max(0, min(n[a] - 1, i));
        idx[a] = i;
        if (d[a] > 0.0) {
            step[a] = 1;
            anext[a] = (lo[a] + (i + 1) * pitch[a] - p1[a]) / d[a];
            dal[a] = pitch[a] / d[a];
        } else if (d[a] < 0.0) {
            step[a] = -1;
            anext[a] = (lo[a] + i * pitch[a] - p1[a]) / d[a];
            dal[a] = -pitch[a] / d[a];
        } else {
            step[a] = 0;
            anext[a] = 1e30;
            dal[a] = 0.0;
        }
    }
    double scale = L;                       // parameter length -> physical length
    if (!(flags & NEFCT_NO_INV_L2)) scale *= (dx_ * dx_) / (L * L);
    e.alpha = (T)amin; e.amax = (T)amax;
    e.ax = (T)anext[0]; e.ay = (T)anext[1]; e.az = (T)anext[2];
    e.dax = (T)dal[0]; e.day = (T)dal[1]; e.daz = (T)dal[2];
    e.i = idx[0]; e.j = idx[1]; e.k = idx[2];
    e.di = step[0]; e.dj = step[1]; e.dk = step[2];
    e.scale = (T)scale;
    e.xdom = fabs(d[0]) >= fabs(d[1]);
    return true;
}

// Visits (voxel index, piece length in parameter units) along the ray.
template <typename T, class Fn>
__device__ __forceinline__ void exact_walk(const GridDev<T> &g, ExactRay<T> e, int su, int sv, int sw, Fn &f)
{
    const int limit = g.nx + g.ny + g.nz + 4;
    for (int it = 0; it < limit; ++it) {
        if (!(e.alpha < e.amax) || (unsigned)e.i >= (unsigned)g.nx || (unsigned)e.j >= (unsigned)g.ny ||
            (unsigned)e.k >= (unsigned)g.nz)
            break;
        const T an = fmin(e.ax, fmin(e.ay, e.az));
        const T aend = fmin(an, e.amax);
        const T len = aend - e.alpha;
        // (u, v) layout: x-dominant rays use the y-fastest copy (su = ny, sv = 1 with u = x)
        const int id = e.xdom ? e.i * su + e.j * sv + e.k * sw : e.j * su + e.i * sv + e.k * sw;
        if (len > (T)0) f(id, len);
        e.alpha = aend;
        if (an == e.ax) { e.i += e.di; e.ax += e.dax; }
        else if (an == e.ay) { e.j += e.dj; e.ay += e.day; }
        else { e.k += e.dk; e.az += e.daz; }
    }
}

template <typename T>
__device__ __forceinline__ T exact_forward(const GridDev<T> &g, const T *r, uint32_t flags, const T *vol, const T *volT)
{
    ExactRay<T> e;
    if (!exact_setup(g, r, flags, e)) return (T)0;
    T acc = (T)0;
    auto f = [&](int id, T len) { acc += __ldg(((e.xdom && volT) ? volT : vol) + id) * len; };
    const int sw = g.nx * g.ny;
    if (e.xdom && volT) exact_walk(g, e, g.ny, 1, sw, f);
    else if (e.xdom) exact_walk(g, e, 1, g.nx, sw, f);
    else exact_walk(g, e, g.nx, 1, sw, f);
    return acc * e.scale;
}

template <typename T>
__device__ __forceinline__ void exact_backward(const GridDev<T> &g, const T *r, uint32_t flags, T y, T *out, T *outT)
{
    ExactRay<T> e;
    if (!exact_setup(g, r, flags, e)) return;
    const T ys = y * e.scale;
    T *base = (e.xdom && outT) ? outT : out;
    auto f = [&](int id, T len) { atomicAdd(base + id, ys * len); };
    const int sw = g.nx * g.ny;
    if (e.xdom && outT) exact_walk(g, e, g.ny, 1, sw, f);
    else if (e.xdom) exact_walk(g, e, 1, g.nx, sw, f);
    else exact_walk(g, e, g.nx, 1, sw, f);
}

// Forward value of one ray: gathers x-driven rays from the y-fastest copy
// volT when there is one, everything else from the x-fastest volume.
template <typename T, bool DIV, bool EXACT = false>
__device__ __forceinline__ T ray_forward(const GridDev<T> &g, const T *r, uint32_t flags, const T *vol, const T *volT)
{
    if (EXACT) return exact_forward(g, r, flags, vol, volT);
    Walk<T> w;
    if (!setup_walk(g, r, flags, w)) return (T)0;
    const int sw = g.nx * g.ny;
    if (!w.xdrive) return gather_walk<T, DIV, true, false>(w, g, vol, g.nx, 1, sw);
    if (volT) return gather_walk<T, DIV, true, false>(w, g, volT, g.ny, 1, sw);
    return gather_walk<T, DIV, false, false>(w, g, vol, 1, g.nx, sw);
}

// Transpose contribution of one ray with value y: x-driven rays reduce into
// the y-fastest accumulator outT when there is one.
template <typename T, bool DIV, bool EXACT = false>
__device__ __forceinline__ void ray_backward(const GridDev<T> &g, const T *r, uint32_t flags, T y, T *out, T *outT)
{
    if (EXACT) {
        exact_backward(g, r, flags, y, out, outT);
        return;
    }
    Walk<T> w;
    if (!setup_walk(g, r, flags, w)) return;
    const int sw = g.nx * g.ny;
    if (!w.xdrive) scatter_walk<T, DIV, true, false>(w, g, out, g.nx, 1, sw, y);
    else if (outT) scatter_walk<T, DIV, true, false>(w, g, outT, g.ny, 1, sw, y);
    else scatter_walk<T, DIV, false, false>(w, g, out, 1, g.nx, sw, y);
}

// out[z][x][y] = in[z][y][x] (32x32 tiles through shared memory)
template <typename T>
__global__ void __launch_bounds__(256) transpose_xy_kernel(const T *__restrict__ in, T *__restrict__ out,
                                                           int nx, int ny)
{
    __shared__ T tile[32][33];
    const size_t plane = (size_t)nx * ny * blockIdx.z;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + threadIdx.x, y = y0 + j;
        if (x < nx && y < ny) tile[j][threadIdx.x] = in[plane + (size_t)y * nx + x];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int y = y0 + threadIdx.x, x = x0 + j;
        if (x < nx && y < ny) out[plane + (size_t)x * ny + y] = tile[threadIdx.x][j];
    }
}

// vol[z][y][x] += accT[z][x][y]
template <typename T>
__global__ void __launch_bounds__(256) fold_add_kernel(const T *__restrict__ accT, T *__restrict__ vol,
                                                       int nx, int ny)
{
    __shared__ T tile[32][33];
    const size_t plane = (size_t)nx * ny * blockIdx.z;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int y = y0 + threadIdx.x, x = x0 + j;
        if (x < nx && y < ny) tile[j][threadIdx.x] = accT[plane + (size_t)x * ny + y];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = x0 + threadIdx.x, y = y0 + j;
        if (x < nx && y < ny) vol[plane + (size_t)y * nx + x] += tile[threadIdx.x][j];
    }
}

}  // namespace nefct
