// Column-warp cone-beam walk (FP32, sm_100a).
//
// The rays of one detector column at one view share their x and y end
// points (the generator's x1, y1, x2, y2 do not depend on the row: the
// source and the column's detector points lie in one vertical plane), so the
// drive axis, pu, pv, kv and every transverse (v) plane position, floor and
// crossing ratio are bit-identical across the rows of a column; only the z
// part (pw, kw, W) differs.
//
// One warp walks 32 consecutive rows of one column in lockstep over the
// union of their slab ranges:
//  * the v part of each slab is computed once per warp: lane j builds the
//    entry of slab kc + j of a 32-slab chunk into the warp's table in shared
//    memory, and every lane reads each slab's entry with one broadcast load;
//    whether the slab crosses a v plane is the same for the whole warp, so
//    the common case without a crossing takes a two-slot split without
//    divergence;
//  * each lane evaluates the z part and the three-voxel split of its own
//    ray exactly as the single-ray walker does (same operations, same order);
//  * the volume (forward) and the accumulator (transpose) are z-fastest
//    copies [y][x][z]: the 32 rows of a warp sit at neighbouring z of the
//    same (u, v) voxel column, so a warp's gather or reduction touches one or
//    two 32-byte sectors instead of one per row band.
// Slabs outside a ray's own range lie outside the grid for that ray and the
// boundary checks reject them; the warp's check-free (interior) range is the
// intersection of its rays' interior ranges.
#pragma once

#include <limits.h>

#include "siddon.cuh"

namespace nefct {


// v part of one slab: biased bases of the low/high v voxel columns (index of
// (k, v, z) = b + floor bits of z), the clamped v floors for the boundary
// checks, and the v crossing ratio.
struct ColEntry {
    unsigned b1, b2;    // k*su + c*sv - 0x4B400000 for the low/high v floor c
    unsigned cv;        // (c1 + 2) | (c2 + 2) << 16, c clamped to [-2, nv + 1]
    float rv;           // crossing ratio, 1 without a v crossing
};

// Warp's table of the slab entries of one 32-slab chunk: .x b1, .y b2,
// .z rv (bits), .w the slab's exit plane offset t + 1 - pu (bits); the
// packed v floors (cv) apart, read by boundary slabs only.
struct ColTable {
    uint4 e[32];
    unsigned cv[32];
};

// Shared (warp-uniform) parameters of the column's walk.
struct ColShared {
    float pu, pv, kv, dv, nv2, nu2;
    int nv;
    unsigned su, sv;
    bool vdiv;
};

// Entry of slab k: planes t = k - nu2 and t + 1, positions and floors as in
// Walker::pos / Walker::next (same operations and order), so every value
// equals the single-ray walker's.  Clamping a floor to [-2, nv + 1] keeps
// every admission decision of the boundary checks.
template <bool DIV> __device__ __forceinline__ ColEntry col_entry(const ColShared &c, int k)
{
    const float ta = __fsub_rn((float)k, c.nu2), tb = __fadd_rn(ta, 1.f);
    auto vpos = [&](float t) {
        float q = __fadd_rn(c.pv, __fmul_rn(c.kv, __fsub_rn(t, c.pu)));
        if (DIV && c.vdiv) q = __fdiv_rn(q, c.dv);
        return __fadd_rn(q, c.nv2);
    };
    const float qa = vpos(ta), qb = vpos(tb);
    const float ma = magic_floor<true>(qa), mb = magic_floor<true>(qb);
    const float q1 = fminf(qa, qb), q2 = fmaxf(qa, qb);
    const float m1 = fminf(ma, mb), m2 = fmaxf(ma, mb);
    ColEntry e;
    e.rv = m1 != m2 ? FP<float>::ratio(__fadd_rn(__fadd_rn(m2, -kFloorMagic), -q1), __fadd_rn(q2, -q1)) : 1.f;
    const int c1 = min(max(__float_as_int(m1) - kFloorMagicBits, -2), c.nv + 1);
    const int c2 = min(max(__float_as_int(m2) - kFloorMagicBits, -2), c.nv + 1);
    const unsigned base = (unsigned)k * c.su - (unsigned)kFloorMagicBits;
    e.b1 = base + (unsigned)c1 * c.sv;
    e.b2 = base + (unsigned)c2 * c.sv;
    e.cv = (unsigned)(c1 + 2) | ((unsigned)(c2 + 2) << 16);
    return e;
}

// Per-lane z state of the walk.
struct ColLane {
    float pw, kw, qaw, maw;
    bool live, up;
};

// Contributions of one slab of a lane's ray: NS slots (voxel index, split
// ratio, activity) in the reference's accumulation order.  In an interior
// slab (CHK false) every slot's index is a voxel of the grid, also for an
// inactive slot (whose ratio is 0: it repeats an active slot's voxel) and
// for a lane without a ray (whose z plane stays at nz/2).
template <int NS, bool CHK> struct ColSlots {
    static constexpr int n = NS;
    static constexpr bool checked = CHK;
    unsigned idx[NS];
    float r[NS];
    bool ok[NS];
};

// One slab of the lane's ray.  WUP: 1 every live ray has kw >= 0, 0 every
// live ray has kw < 0, 2 mixed (per-lane choice).  The v crossing is shared
// by the warp (b1 != b2): without one (VX false) the split has two slots,
// (v1, w1) with ratio rw and (v1, w2) with 1 - rw, which is the general
// three-slot split with rv = 1 (its third ratio, 1 - max(rv, rw), is 0 and
// its slot inactive); with one, the general split.  SPLIT 0 takes the
// general split for every slab (no branch: the forward's loads of
// consecutive slabs interleave better); 1 the two-slot split; 2 the same
// with the second slot always at w2 (it differs from the reference's pairing
// only when the ratio rounds to 1 or above, where that slot's weight is a
// rounding error; for the float transpose, whose atomic sums are not
// reproducible anyway).  f(slots) consumes.  The slab's table entry (b1,
// b2, exit plane offset d, v ratio rv, packed v floors cv) comes from the
// caller; TWO: the two-slot split (the caller's SPLIT and no v crossing).
template <bool DIV, bool CHECK, int WUP, int SPLIT, bool TWO, class Fn>
__device__ __forceinline__ void col_lane_slab(ColLane &L, float dz, bool zdiv, float nz2, int nv, int nz,
                                              unsigned b1, unsigned b2, float d, float rv, unsigned cv, Fn &f)
{
    float qbw = __fadd_rn(L.pw, __fmul_rn(L.kw, d));
    if (DIV && zdiv) qbw = __fdiv_rn(qbw, dz);
    qbw = __fadd_rn(qbw, nz2);
    const float mbw = magic_floor<CHECK>(qbw);
    const bool up = WUP == 2 ? L.up : WUP == 1;
    const float q1w = up ? L.qaw : qbw, q2w = up ? qbw : L.qaw;
    const float m1w = up ? L.maw : mbw, m2w = up ? mbw : L.maw;
    L.qaw = qbw;
    L.maw = mbw;
    const bool wx = m1w != m2w;
    const float rw = wx ? FP<float>::ratio(__fadd_rn(__fadd_rn(m2w, -kFloorMagic), -q1w), __fadd_rn(q2w, -q1w)) : 1.f;
    const unsigned i1 = (unsigned)__float_as_int(m1w), i2 = (unsigned)__float_as_int(m2w);
    const int cv1 = CHECK ? (int)(cv & 0xffffu) - 2 : 0, cv2 = CHECK ? (int)(cv >> 16) - 2 : 0;
    const int cw1 = (int)i1 - kFloorMagicBits, cw2 = (int)i2 - kFloorMagicBits;
    if constexpr (TWO) {
        // no v crossing (uniform across the warp)
        const bool vfirst = 1.f > rw;
        ColSlots<2, CHECK> s;
        s.r[0] = rw;                            // min(1, rw)
        s.r[1] = __fsub_rn(1.f, rw);            // |1 - rw|
        s.idx[0] = b1 + i1;
        s.idx[1] = b1 + ((SPLIT == 2 || vfirst) ? i2 : i1);
        if (CHECK) {
            const bool adm = L.live && (unsigned)cv1 < (unsigned)nv && (unsigned)(cw1 + (int)wx) < (unsigned)(nz + (int)wx);
            const int mw = (SPLIT == 2 || vfirst) ? cw2 : cw1;     // the slot's own voxel
            s.ok[0] = adm && cw1 >= 0;
            s.ok[1] = adm && wx && (unsigned)mw < (unsigned)nz;
        } else {
            s.ok[0] = L.live;
            s.ok[1] = L.live && wx;
        }
        f(s);
    } else {
        const bool vx = SPLIT || b1 != b2;
        const bool vfirst = rv > rw;
        ColSlots<3, CHECK> s;
        s.r[0] = fminf(rv, rw);
        s.r[1] = fabsf(__fsub_rn(rv, rw));
        s.r[2] = __fsub_rn(1.f, fmaxf(rv, rw));
        s.idx[0] = b1 + i1;
        s.idx[1] = vfirst ? b1 + i2 : b2 + i1;
        s.idx[2] = b2 + i2;
        if (CHECK) {
            // slab admission (reference siddon.cu.cc :80, :92, :112, :116, :132)
            const bool adm = L.live && (unsigned)(cv1 + (int)vx) < (unsigned)(nv + (int)vx) &&
                             (unsigned)(cw1 + (int)wx) < (unsigned)(nz + (int)wx);
            const int mv = vfirst ? cv1 : cv2, mw = vfirst ? cw2 : cw1;
            s.ok[0] = adm && (cv1 | cw1) >= 0;
            s.ok[1] = adm && (vx || wx) && (unsigned)mv < (unsigned)nv && (unsigned)mw < (unsigned)nz;
            s.ok[2] = adm && vx && wx && cv2 < nv && cw2 < nz;
        } else {
            s.ok[0] = L.live;
            s.ok[1] = L.live && (vx || wx);
            s.ok[2] = L.live && vx && wx;
        }
        f(s);
    }
}

// One slab of the lane's one ray, its entry read from the warp's table.
template <bool DIV, bool CHECK, int WUP, int SPLIT, class Fn>
__device__ __forceinline__ void col_slab(ColLane &L, float dz, bool zdiv, float nz2, int nv, int nz,
                                         const ColTable &tab, int j, Fn &f)
{
    const uint4 te = tab.e[j];          // same address for every lane: one broadcast
    const unsigned cv = CHECK ? tab.cv[j] : 0u;
    if (SPLIT && te.x == te.y)
        col_lane_slab<DIV, CHECK, WUP, SPLIT, true>(L, dz, zdiv, nz2, nv, nz, te.x, te.y, __uint_as_float(te.w),
                                                    __uint_as_float(te.z), cv, f);
    else
        col_lane_slab<DIV, CHECK, WUP, SPLIT, false>(L, dz, zdiv, nz2, nv, nz, te.x, te.y, __uint_as_float(te.w),
                                                     __uint_as_float(te.z), cv, f);
}

// The same slab for the R rays of a lane (rows l, l + 32, ... of the
// column): one table read and one split decision for all of them;
// f(slots, r) consumes ray r's slots.
template <bool DIV, bool CHECK, int WUP, int SPLIT, int R, class Fn>
__device__ __forceinline__ void col_slab_rows(ColLane (&L)[R], float dz, bool zdiv, float nz2, int nv, int nz,
                                              const ColTable &tab, int j, Fn &f)
{
    const uint4 te = tab.e[j];
    const unsigned cv = CHECK ? tab.cv[j] : 0u;
    const float d = __uint_as_float(te.w), rv = __uint_as_float(te.z);
    if (SPLIT && te.x == te.y) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            auto fr = [&](const auto &s) { f(s, r); };
            col_lane_slab<DIV, CHECK, WUP, SPLIT, true>(L[r], dz, zdiv, nz2, nv, nz, te.x, te.y, d, rv, cv, fr);
        }
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            auto fr = [&](const auto &s) { f(s, r); };
            col_lane_slab<DIV, CHECK, WUP, SPLIT, false>(L[r], dz, zdiv, nz2, nv, nz, te.x, te.y, d, rv, cv, fr);
        }
    }
}

// Walks slabs [a, b] (inside the current 32-slab chunk starting at kc) in
// one check mode.
template <bool DIV, bool CHECK, int WUP, int SPLIT, class Fn>
__device__ __forceinline__ void col_range(int a, int b, int kc, const ColShared &c, ColLane &L,
                                          const ColTable &tab, const GridDev<float> &g, Fn &f)
{
    const bool zdiv = g.dz != 1.f;
#pragma unroll 4
    for (int k = a; k <= b; ++k)
        col_slab<DIV, CHECK, WUP, SPLIT>(L, g.dz, zdiv, g.nz2, c.nv, g.nz, tab, k - kc, f);
}

// Slabs [K0, K1] of the warp in 32-slab chunks (lane j builds the entry of
// slab kc + j into the warp's table); boundary slabs outside [KI0, KI1] with
// range checks.  The slab planes k - nu2 and k + 1 - nu2 are exact (nu2 is a
// multiple of 1/2 and |k| < 2^22), so the table's exit plane offset equals
// the one a walk carrying t += 1 evaluates.
template <bool DIV, int WUP, int SPLIT, class Fn>
__device__ __forceinline__ void col_walk(const ColShared &c, ColLane &L, int K0, int K1, int KI0, int KI1,
                                         const GridDev<float> &g, ColTable &tab, Fn &f)
{
    // plane K0 - nu2 (entry plane of the first slab)
    const float t = __fsub_rn((float)K0, c.nu2);
    float q = __fadd_rn(L.pw, __fmul_rn(L.kw, __fsub_rn(t, c.pu)));
    if (DIV && g.dz != 1.f) q = __fdiv_rn(q, g.dz);
    L.qaw = __fadd_rn(q, g.nz2);
    L.maw = magic_floor<true>(L.qaw);
    const int lane = threadIdx.x & 31;
    if (KI0 > KI1) { KI0 = K1 + 1; KI1 = K1; }      // no interior: everything checked
    for (int kc = K0; kc <= K1; kc += 32) {
        const ColEntry e = col_entry<DIV>(c, kc + lane);
        const float d = __fsub_rn(__fadd_rn(__fsub_rn((float)(kc + lane), c.nu2), 1.f), c.pu);
        __syncwarp();                   // the previous chunk's reads are done
        tab.e[lane] = make_uint4(e.b1, e.b2, __float_as_uint(e.rv), __float_as_uint(d));
        tab.cv[lane] = e.cv;
        __syncwarp();
        const int ke = min(K1, kc + 31);
        col_range<DIV, true, WUP, SPLIT>(kc, min(ke, KI0 - 1), kc, c, L, tab, g, f);
        col_range<DIV, false, WUP, SPLIT>(max(kc, KI0), min(ke, KI1), kc, c, L, tab, g, f);
        col_range<DIV, true, WUP, SPLIT>(max(kc, KI1 + 1), ke, kc, c, L, tab, g, f);
    }
}

template <bool DIV, int SPLIT, class Fn>
__device__ __forceinline__ void col_walk_any(const ColShared &c, ColLane &L, int K0, int K1, int KI0, int KI1,
                                             const GridDev<float> &g, Fn &f)
{
    // one table per warp; column-warp blocks are 32 x (at most 8) threads
    __shared__ ColTable tables[8];
    ColTable &tab = tables[threadIdx.y];
    const bool all_up = __all_sync(0xffffffffu, L.up || !L.live);
    const bool all_down = __all_sync(0xffffffffu, !L.up || !L.live);
    if (all_up) col_walk<DIV, 1, SPLIT>(c, L, K0, K1, KI0, KI1, g, tab, f);
    else if (all_down) col_walk<DIV, 0, SPLIT>(c, L, K0, K1, KI0, KI1, g, tab, f);
    else col_walk<DIV, 2, SPLIT>(c, L, K0, K1, KI0, KI1, g, tab, f);
}

// Strides of the z-fastest layout [y][x][z] along (u, v) of the drive axis.
__device__ __forceinline__ void col_strides(const GridDev<float> &g, bool xdrive, unsigned &su, unsigned &sv)
{
    const unsigned xs = (unsigned)g.nz, ys = (unsigned)g.nx * (unsigned)g.nz;
    su = xdrive ? xs : ys;
    sv = xdrive ? ys : xs;
}

// Sets up the warp: shared parameters from the first live lane, the warp's
// slab and interior ranges.  Returns false when the rays do not share their
// v parameters bit for bit (each lane then walks alone).
__device__ __forceinline__ bool col_setup(const GridDev<float> &g, const Walk<float> &w, bool live, ColShared &c,
                                          ColLane &L, int &K0, int &K1, int &KI0, int &KI1)
{
    const unsigned lm = __ballot_sync(0xffffffffu, live);
    const int src = __ffs(lm) - 1;
    c.pu = __shfl_sync(0xffffffffu, w.pu, src);
    c.pv = __shfl_sync(0xffffffffu, w.pv, src);
    c.kv = __shfl_sync(0xffffffffu, w.kv, src);
    const bool xdrive = __shfl_sync(0xffffffffu, (int)w.xdrive, src) != 0;
    const bool same = !live || (__float_as_int(w.pu) == __float_as_int(c.pu) &&
                                __float_as_int(w.pv) == __float_as_int(c.pv) &&
                                __float_as_int(w.kv) == __float_as_int(c.kv) && w.xdrive == xdrive);
    if (!__all_sync(0xffffffffu, same)) return false;
    c.dv = xdrive ? g.dy : 1.f;
    c.vdiv = xdrive && g.dy != 1.f;
    c.nv2 = xdrive ? g.ny2 : g.nx2;
    c.nu2 = xdrive ? g.nx2 : g.ny2;
    c.nv = xdrive ? g.ny : g.nx;
    col_strides(g, xdrive, c.su, c.sv);
    K0 = __reduce_min_sync(0xffffffffu, live ? w.k0 : INT_MAX);
    K1 = __reduce_max_sync(0xffffffffu, live ? w.k1 : INT_MIN);
    KI0 = __reduce_max_sync(0xffffffffu, live ? w.ki0 : INT_MIN);
    KI1 = __reduce_min_sync(0xffffffffu, live ? w.ki1 : INT_MAX);
    // a lane without a ray walks the plane z = nz/2 (indices stay in the grid)
    L.pw = live ? w.pw : 0.f;
    L.kw = live ? w.kw : 0.f;
    L.live = live;
    L.up = w.kw >= 0.f;
    return true;
}

// ---- R rays per lane: rows l, l + 32, ..., l + 32 (R - 1) of the column ----
//
// The warp's table serves 32 R rays: each slab's entry is read and its split
// decided once per lane for all of them.  Each ray's own arithmetic is the
// one-ray walk's.

template <bool DIV, bool CHECK, int WUP, int SPLIT, int R, class Fn>
__device__ __forceinline__ void col_range_rows(int a, int b, int kc, const ColShared &c, ColLane (&L)[R],
                                               const ColTable &tab, const GridDev<float> &g, Fn &f)
{
    const bool zdiv = g.dz != 1.f;
#pragma unroll 2
    for (int k = a; k <= b; ++k)
        col_slab_rows<DIV, CHECK, WUP, SPLIT, R>(L, g.dz, zdiv, g.nz2, c.nv, g.nz, tab, k - kc, f);
}

template <bool DIV, int WUP, int SPLIT, int R, class Fn>
__device__ __forceinline__ void col_walk_rows(const ColShared &c, ColLane (&L)[R], int K0, int K1, int KI0, int KI1,
                                              const GridDev<float> &g, ColTable &tab, Fn &f)
{
    const float t = __fsub_rn((float)K0, c.nu2);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        float q = __fadd_rn(L[r].pw, __fmul_rn(L[r].kw, __fsub_rn(t, c.pu)));
        if (DIV && g.dz != 1.f) q = __fdiv_rn(q, g.dz);
        L[r].qaw = __fadd_rn(q, g.nz2);
        L[r].maw = magic_floor<true>(L[r].qaw);
    }
    const int lane = threadIdx.x & 31;
    if (KI0 > KI1) { KI0 = K1 + 1; KI1 = K1; }
    for (int kc = K0; kc <= K1; kc += 32) {
        const ColEntry e = col_entry<DIV>(c, kc + lane);
        const float d = __fsub_rn(__fadd_rn(__fsub_rn((float)(kc + lane), c.nu2), 1.f), c.pu);
        __syncwarp();
        tab.e[lane] = make_uint4(e.b1, e.b2, __float_as_uint(e.rv), __float_as_uint(d));
        tab.cv[lane] = e.cv;
        __syncwarp();
        const int ke = min(K1, kc + 31);
        col_range_rows<DIV, true, WUP, SPLIT, R>(kc, min(ke, KI0 - 1), kc, c, L, tab, g, f);
        col_range_rows<DIV, false, WUP, SPLIT, R>(max(kc, KI0), min(ke, KI1), kc, c, L, tab, g, f);
        col_range_rows<DIV, true, WUP, SPLIT, R>(max(kc, KI1 + 1), ke, kc, c, L, tab, g, f);
    }
}

template <bool DIV, int SPLIT, int R, class Fn>
__device__ __forceinline__ void col_walk_any_rows(const ColShared &c, ColLane (&L)[R], int K0, int K1, int KI0,
                                                  int KI1, const GridDev<float> &g, Fn &f)
{
    __shared__ ColTable tables[8];
    ColTable &tab = tables[threadIdx.y];
    bool up = true, down = true;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        up = up && (L[r].up || !L[r].live);
        down = down && (!L[r].up || !L[r].live);
    }
    const bool all_up = __all_sync(0xffffffffu, up), all_down = __all_sync(0xffffffffu, down);
    if (all_up) col_walk_rows<DIV, 1, SPLIT, R>(c, L, K0, K1, KI0, KI1, g, tab, f);
    else if (all_down) col_walk_rows<DIV, 0, SPLIT, R>(c, L, K0, K1, KI0, KI1, g, tab, f);
    else col_walk_rows<DIV, 2, SPLIT, R>(c, L, K0, K1, KI0, KI1, g, tab, f);
}

// col_setup for R rays per lane (all in one detector column).
template <int R>
__device__ __forceinline__ bool col_setup_rows(const GridDev<float> &g, const Walk<float> (&w)[R],
                                               const bool (&live)[R], ColShared &c, ColLane (&L)[R], int &K0,
                                               int &K1, int &KI0, int &KI1)
{
    bool any = false;
    int first = 0;
#pragma unroll
    for (int r = R - 1; r >= 0; --r)
        if (live[r]) { any = true; first = r; }
    float pu = w[0].pu, pv = w[0].pv, kv = w[0].kv;
    bool xd = w[0].xdrive;
#pragma unroll
    for (int r = 1; r < R; ++r)
        if (first == r) { pu = w[r].pu; pv = w[r].pv; kv = w[r].kv; xd = w[r].xdrive; }
    const unsigned lm = __ballot_sync(0xffffffffu, any);
    const int src = __ffs(lm) - 1;
    c.pu = __shfl_sync(0xffffffffu, pu, src);
    c.pv = __shfl_sync(0xffffffffu, pv, src);
    c.kv = __shfl_sync(0xffffffffu, kv, src);
    const bool xdrive = __shfl_sync(0xffffffffu, (int)xd, src) != 0;
    bool same = true;
    int k0 = INT_MAX, k1 = INT_MIN, ki0 = INT_MIN, ki1 = INT_MAX;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        same = same && (!live[r] || (__float_as_int(w[r].pu) == __float_as_int(c.pu) &&
                                     __float_as_int(w[r].pv) == __float_as_int(c.pv) &&
                                     __float_as_int(w[r].kv) == __float_as_int(c.kv) && w[r].xdrive == xdrive));
        if (live[r]) {
            k0 = min(k0, w[r].k0);
            k1 = max(k1, w[r].k1);
            ki0 = max(ki0, w[r].ki0);
            ki1 = min(ki1, w[r].ki1);
        }
    }
    if (!__all_sync(0xffffffffu, same)) return false;
    c.dv = xdrive ? g.dy : 1.f;
    c.vdiv = xdrive && g.dy != 1.f;
    c.nv2 = xdrive ? g.ny2 : g.nx2;
    c.nu2 = xdrive ? g.nx2 : g.ny2;
    c.nv = xdrive ? g.ny : g.nx;
    col_strides(g, xdrive, c.su, c.sv);
    K0 = __reduce_min_sync(0xffffffffu, k0);
    K1 = __reduce_max_sync(0xffffffffu, k1);
    KI0 = __reduce_max_sync(0xffffffffu, ki0);
    KI1 = __reduce_min_sync(0xffffffffu, ki1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        L[r].pw = live[r] ? w[r].pw : 0.f;
        L[r].kw = live[r] ? w[r].kw : 0.f;
        L[r].live = live[r];
        L[r].up = w[r].kw >= 0.f;
    }
    return true;
}

}  // namespace nefct
