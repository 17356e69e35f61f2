// force_device.cuh -- device code of the i-block x j-particle direct sum,
// shared by the launch-per-call kernels (force.cu) and the resident serving
// kernel (resident.cu): per-i register state, the pair terms, one j-tile's
// consumption, and one task (an i-tile against a j-split) with its bulk-copy
// pipeline and its epilogue.  The pair terms' reference and the work
// decomposition are described at the top of force.cu.
#pragma once
#include <cfloat>
#include "common.cuh"
#include "kernels.h"

namespace g6 {

constexpr uint64_t kWaitLimitNs = 1000000000ull;  // 1 s per tile wait
#ifndef G6B200_FOLD_TERMS
#define G6B200_FOLD_TERMS 64
#endif
constexpr int kFlush = G6B200_FOLD_TERMS;         // FP32 terms per FP64 fold
constexpr int kMaxWarps = 8;

// T j per shared-memory tile, held as U records of JPU j each.
template <int K> struct Traits;
template <> struct Traits<kKernMixedDS> {
    using JRec = JRecMixed;
    static constexpr int T = 256, JPU = 1, U = T;
};
template <> struct Traits<kKernMixedP> {
    using JRec = JPairMixed;
    static constexpr int T = 256, JPU = 2, U = T / 2;
};
template <> struct Traits<kKernF64> {
    using JRec = JRecF64;
    static constexpr int T = 128, JPU = 1, U = T;
};

// Per-i register state.

struct StateMixedBase {
    float vx, vy, vz, h2;
    float ax, ay, az, jx, jy, jz, pt;   // FP32 sums since the last fold
    double Ax, Ay, Az, Jx, Jy, Jz, Pt;  // FP64 totals
    float nr2;                          // best r^2 so far
    int nj, idx, i;
};

struct StateMixed : StateMixedBase {
    float xh, yh, zh, xl, yl, zl;
};

struct StateF64 {
    double x, y, z, vx, vy, vz, h2;
    double eps2;  // per-i softening (GRAPE-4 variant only)
    double Ax, Ay, Az, Jx, Jy, Jz, Pt;
    double nr2;
    int nj, idx, i;
};

template <int K> struct StateOf;
template <> struct StateOf<kKernMixedDS> { using type = StateMixed; };
template <> struct StateOf<kKernF64> { using type = StateF64; };

__device__ __forceinline__ void nb_push(const ForceParams &p, int i, int j) {
    int k = atomicAdd(&p.nb_count[i], 1);
    if (k < p.nb_cap) p.nb_list[(size_t)i * p.nb_cap + k] = j;
}

__device__ __forceinline__ void init_mixed(StateMixedBase &s, const IRec &q) {
    s.vx = (float)q.v[0];
    s.vy = (float)q.v[1];
    s.vz = (float)q.v[2];
    s.h2 = (float)q.h2;
    s.idx = q.index;
    s.ax = s.ay = s.az = s.jx = s.jy = s.jz = s.pt = 0.f;
    s.Ax = s.Ay = s.Az = s.Jx = s.Jy = s.Jz = s.Pt = 0.0;
    s.nr2 = FLT_MAX;
    s.nj = -1;
}

__device__ __forceinline__ void load_i(StateMixed &s, const IRec &q, const ForceParams &p, bool &range_ok) {
    range_ok &= to_fixed_split(q.x[0], p.fs, s.xh, s.xl);
    range_ok &= to_fixed_split(q.x[1], p.fs, s.yh, s.yl);
    range_ok &= to_fixed_split(q.x[2], p.fs, s.zh, s.zl);
    init_mixed(s, q);
}

__device__ __forceinline__ void load_i(StateF64 &s, const IRec &q, const ForceParams &, bool &) {
    s.x = q.x[0];
    s.y = q.x[1];
    s.z = q.x[2];
    s.vx = q.v[0];
    s.vy = q.v[1];
    s.vz = q.v[2];
    s.h2 = q.h2;
    s.idx = q.index;
    s.Ax = s.Ay = s.Az = s.Jx = s.Jy = s.Jz = s.Pt = 0.0;
    s.nr2 = DBL_MAX;
    s.nj = -1;
}

// A j-particle as the mixed kernels see it after the shared-memory load.
struct JMixed {
    float dx, dy, dz;  // exact position difference rounded to FP32
    float vx, vy, vz, m;
    int index;
};

__device__ __forceinline__ void diff(const StateMixed &s, const JRecMixed &J, JMixed &o) {
    const float4 hi = J.hi, lo = J.lo, ve = J.vel;
    o.dx = (hi.x - s.xh) + (lo.x - s.xl);
    o.dy = (hi.y - s.yh) + (lo.y - s.yl);
    o.dz = (hi.z - s.zh) + (lo.z - s.zl);
    o.vx = ve.x;
    o.vy = ve.y;
    o.vz = ve.z;
    o.m = hi.w;
    o.index = __float_as_int(lo.w);
}

template <bool CHK, bool NB, bool IDENT, class S>
__device__ __forceinline__ void interact_mixed(S &s, const JMixed &J, int jg, float eps2, const ForceParams &p) {
    const float dvx = J.vx - s.vx;
    const float dvy = J.vy - s.vy;
    const float dvz = J.vz - s.vz;
    const float r2n = fmaf(J.dz, J.dz, fmaf(J.dy, J.dy, J.dx * J.dx));
    const float rv = fmaf(J.dz, dvz, fmaf(J.dy, dvy, J.dx * dvx));
    float r2 = r2n + eps2;
    float mj = J.m;
    float r2nn = r2n;
    bool self = false;
    if (CHK) {
        self = IDENT ? (jg == s.idx) : (J.index == s.idx);
        r2 = self ? 1.f : r2;
        mj = self ? 0.f : mj;
        r2nn = self ? FLT_MAX : r2nn;
    }
    float y = rsqrt_approx(r2);
    // One Newton-Raphson step: y <- y (1.5 - 0.5 r2 y^2).
    const float hy = (0.5f * r2) * y;
    y = y * fmaf(-hy, y, 1.5f);
    const float r2inv = y * y;
    const float mr = mj * y;
    const float mr3 = mr * r2inv;
    const float a3 = -3.f * rv * r2inv;
    s.pt -= mr;
    s.ax = fmaf(mr3, J.dx, s.ax);
    s.ay = fmaf(mr3, J.dy, s.ay);
    s.az = fmaf(mr3, J.dz, s.az);
    s.jx = fmaf(mr3, fmaf(a3, J.dx, dvx), s.jx);
    s.jy = fmaf(mr3, fmaf(a3, J.dy, dvy), s.jy);
    s.jz = fmaf(mr3, fmaf(a3, J.dz, dvz), s.jz);
    if (r2nn < s.nr2) {
        s.nr2 = r2nn;
        s.nj = jg;
    }
    if (NB) {
        bool hit = CHK && self ? (p.include_self && s.h2 > 0.f) : (r2n < s.h2);
        if (hit) nb_push(p, s.i, jg);
    }
}

template <bool CHK, bool NB, bool IDENT, bool G4 = false, bool PO = false>
__device__ __forceinline__ void interact(StateF64 &s, const double4 &pos, const double4 &vel,
                                         int jg, double eps2, const ForceParams &p) {
    if constexpr (PO) {
        // Potential only: the pot term of the full form below.
        const double dx = pos.x - s.x;
        const double dy = pos.y - s.y;
        const double dz = pos.z - s.z;
        double r2 = dx * dx + dy * dy + dz * dz + eps2;
        double mj = pos.w;
        if (CHK) {
            const bool self = IDENT ? (jg == s.idx) : ((int)vel.w == s.idx);
            r2 = self ? 1.0 : r2;
            mj = self ? 0.0 : mj;
        }
        s.Pt -= mj * rsqrt(r2);
        return;
    }
    const double dx = pos.x - s.x;
    const double dy = pos.y - s.y;
    const double dz = pos.z - s.z;
    const double dvx = vel.x - s.vx;
    const double dvy = vel.y - s.vy;
    const double dvz = vel.z - s.vz;
    const double rv = dx * dvx + dy * dvy + dz * dvz;
    if (G4) {
        // The same rounding sequence as g4_r2() in the neighbour-list pass.
        double r2 = g4_r2(dx, dy, dz, s.eps2);
        if (NB && r2 < s.h2) nb_push(p, s.i, jg);
        const bool zero = !(r2 > 0.0);
        const double mj = zero ? 0.0 : pos.w;
        const double r2nn = zero ? DBL_MAX : r2;
        r2 = zero ? 1.0 : r2;
        const double rinv = rsqrt(r2);
        const double r2inv = rinv * rinv;
        const double mr = mj * rinv;
        const double mr3 = mr * r2inv;
        const double a3 = -3.0 * rv * r2inv;
        s.Pt -= mr;
        s.Ax += mr3 * dx;
        s.Ay += mr3 * dy;
        s.Az += mr3 * dz;
        s.Jx += mr3 * (dvx + a3 * dx);
        s.Jy += mr3 * (dvy + a3 * dy);
        s.Jz += mr3 * (dvz + a3 * dz);
        if (r2nn < s.nr2) {
            s.nr2 = r2nn;
            s.nj = jg;
        }
        return;
    }
    const double r2n = dx * dx + dy * dy + dz * dz;
    double r2 = r2n + eps2;
    double mj = pos.w;
    double r2nn = r2n;
    bool self = false;
    if (CHK) {
        self = IDENT ? (jg == s.idx) : ((int)vel.w == s.idx);
        r2 = self ? 1.0 : r2;
        mj = self ? 0.0 : mj;
        r2nn = self ? DBL_MAX : r2nn;
    }
    const double rinv = rsqrt(r2);
    const double r2inv = rinv * rinv;
    const double mr = mj * rinv;
    const double mr3 = mr * r2inv;
    const double a3 = -3.0 * rv * r2inv;
    s.Pt -= mr;
    s.Ax += mr3 * dx;
    s.Ay += mr3 * dy;
    s.Az += mr3 * dz;
    s.Jx += mr3 * (dvx + a3 * dx);
    s.Jy += mr3 * (dvy + a3 * dy);
    s.Jz += mr3 * (dvz + a3 * dz);
    if (r2nn < s.nr2) {
        s.nr2 = r2nn;
        s.nj = jg;
    }
    if (NB) {
        bool hit = CHK && self ? (p.include_self && s.h2 > 0.0) : (r2n < s.h2);
        if (hit) nb_push(p, s.i, jg);
    }
}

// ---- paired layout: one FP32x2 instruction evaluates i against two j.
// i-side values are held negated and duplicated in both halves, so every
// difference is an FP32x2 add of a j-pair and a loop-invariant register pair.
struct StateMixedP {
    float2 nxh, nyh, nzh, nxl, nyl, nzl, nvx, nvy, nvz;
    float h2;
    float2 ax, ay, az, jx, jy, jz, pm;  // FP32 sums since the last fold; pm = sum m/(4r)
    unsigned qa;                        // error indicators (kVarStats): bits of max m/(2r^2) (unsigned max)
    int qj;                             // and of max m/r^3 (signed max: the self term's -0.0 never wins)
    double Ax, Ay, Az, Jx, Jy, Jz, Pt;
    float nr2;
    int nj, idx, i;
};
template <> struct StateOf<kKernMixedP> { using type = StateMixedP; };

__device__ __forceinline__ float2 dup(float v) { return make_float2(v, v); }

__device__ __forceinline__ void load_i(StateMixedP &s, const IRec &q, const ForceParams &p, bool &range_ok) {
    float h, l;
    range_ok &= to_fixed_split(q.x[0], p.fs, h, l);
    s.nxh = dup(-h);
    s.nxl = dup(-l);
    range_ok &= to_fixed_split(q.x[1], p.fs, h, l);
    s.nyh = dup(-h);
    s.nyl = dup(-l);
    range_ok &= to_fixed_split(q.x[2], p.fs, h, l);
    s.nzh = dup(-h);
    s.nzl = dup(-l);
    s.nvx = dup(-(float)q.v[0]);
    s.nvy = dup(-(float)q.v[1]);
    s.nvz = dup(-(float)q.v[2]);
    s.h2 = (float)q.h2;
    s.idx = q.index;
    s.ax = s.ay = s.az = s.jx = s.jy = s.jz = s.pm = make_float2(0.f, 0.f);
    s.qa = 0u;
    s.qj = 0;
    s.Ax = s.Ay = s.Az = s.Jx = s.Jy = s.Jz = s.Pt = 0.0;
    s.nr2 = FLT_MAX;
    s.nj = -1;
}

template <bool CHK, bool NB, bool IDENT, bool PO = false, bool STATS = false>
__device__ __forceinline__ void interact_pair(StateMixedP &s, const JPairMixed &J, int jg0, float2 eps2,
                                              const ForceParams &p) {
    if constexpr (PO) {
        // Potential only: the exact position difference, r^2, the refined
        // inverse distance and m/r -- the pot terms of the full form below,
        // rounded identically.
        const float2 dx = __fadd2_rn(__fadd2_rn(make_float2(J.hxy.x, J.hxy.y), s.nxh),
                                     __fadd2_rn(make_float2(J.lxy.x, J.lxy.y), s.nxl));
        const float2 dy = __fadd2_rn(__fadd2_rn(make_float2(J.hxy.z, J.hxy.w), s.nyh),
                                     __fadd2_rn(make_float2(J.lxy.z, J.lxy.w), s.nyl));
        const float2 dz = __fadd2_rn(__fadd2_rn(make_float2(J.hzm.x, J.hzm.y), s.nzh),
                                     __fadd2_rn(make_float2(J.lzi.x, J.lzi.y), s.nzl));
        float2 r2 = __fadd2_rn(__ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx))), eps2);
        float2 m = make_float2(J.hzm.z, J.hzm.w);
        if (CHK) {
            const bool self0 = IDENT ? (jg0 == s.idx) : (__float_as_int(J.lzi.z) == s.idx);
            const bool self1 = IDENT ? (jg0 + 1 == s.idx) : (__float_as_int(J.lzi.w) == s.idx);
            r2.x = self0 ? 1.f : r2.x;
            r2.y = self1 ? 1.f : r2.y;
            m.x = self0 ? 0.f : m.x;
            m.y = self1 ? 0.f : m.y;
        }
        float2 y = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
        const float2 ry = __fmul2_rn(r2, y);
        y = __fmul2_rn(y, __ffma2_rn(ry, y, dup(-3.f)));
        s.pm = __fadd2_rn(s.pm, __fmul2_rn(m, y));
        return;
    }
    const float2 dx = __fadd2_rn(__fadd2_rn(make_float2(J.hxy.x, J.hxy.y), s.nxh),
                                 __fadd2_rn(make_float2(J.lxy.x, J.lxy.y), s.nxl));
    const float2 dy = __fadd2_rn(__fadd2_rn(make_float2(J.hxy.z, J.hxy.w), s.nyh),
                                 __fadd2_rn(make_float2(J.lxy.z, J.lxy.w), s.nyl));
    const float2 dz = __fadd2_rn(__fadd2_rn(make_float2(J.hzm.x, J.hzm.y), s.nzh),
                                 __fadd2_rn(make_float2(J.lzi.x, J.lzi.y), s.nzl));
    const float2 dvx = __fadd2_rn(make_float2(J.vxy.x, J.vxy.y), s.nvx);
    const float2 dvy = __fadd2_rn(make_float2(J.vxy.z, J.vxy.w), s.nvy);
    const float2 dvz = __fadd2_rn(make_float2(J.vz.x, J.vz.y), s.nvz);
    const float2 r2n = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    const float2 rv = __ffma2_rn(dz, dvz, __ffma2_rn(dy, dvy, __fmul2_rn(dx, dvx)));
    float2 r2 = __fadd2_rn(r2n, eps2);
    float2 m = make_float2(J.hzm.z, J.hzm.w);
    float2 r2nn = r2n;
    bool self0 = false, self1 = false;
    if (CHK) {
        self0 = IDENT ? (jg0 == s.idx) : (__float_as_int(J.lzi.z) == s.idx);
        self1 = IDENT ? (jg0 + 1 == s.idx) : (__float_as_int(J.lzi.w) == s.idx);
        r2.x = self0 ? 1.f : r2.x;
        r2.y = self1 ? 1.f : r2.y;
        m.x = self0 ? 0.f : m.x;
        m.y = self1 ? 0.f : m.y;
        r2nn.x = self0 ? FLT_MAX : r2nn.x;
        r2nn.y = self1 ? FLT_MAX : r2nn.y;
    }
    float2 y = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    // One Newton-Raphson step, kept at -2 times its value:
    // y' = y (r2 y^2 - 3) = -2 y (1.5 - 0.5 r2 y^2), one instruction fewer
    // than the textbook form.  Every product below is the scalar kernel's
    // scaled by a power of two (exact), and the record's mass is -m/8, so
    // mr3 = (-m/8)(-2y)(4 y^2) and a3 = (-0.75 rv)(4 y^2) come out
    // bit-identical to the textbook form; pm sums m/(4r).
    const float2 ry = __fmul2_rn(r2, y);
    y = __fmul2_rn(y, __ffma2_rn(ry, y, dup(-3.f)));
    const float2 r2inv = __fmul2_rn(y, y);
    const float2 mr = __fmul2_rn(m, y);
    const float2 mr3 = __fmul2_rn(mr, r2inv);
    const float2 a3 = __fmul2_rn(__fmul2_rn(rv, dup(-0.75f)), r2inv);
    if (STATS) {
        // The refinement's error indicators, the largest single terms:
        // mr y = -m/(2 r^2) (y is -2/r, see above) and mr3 = m/r^3.  The
        // maxima are integer maxima of the bit patterns, off the FMA pipe:
        // non-positive floats order like their bits read as unsigned (t),
        // non-negative ones like their bits read as signed (mr3).  The self
        // term (m = +0, y < 0) gives mr3 = -0.0, whose bits 0x80000000 would
        // win an unsigned maximum over every positive float; as a signed
        // int it is the smallest value.
        // Both halves of the pair go into one register per indicator with a
        // three-input maximum.
        const float2 t = __fmul2_rn(mr, y);
        s.qa = __vimax3_u32(s.qa, __float_as_uint(t.x), __float_as_uint(t.y));
        s.qj = __vimax3_s32(s.qj, __float_as_int(mr3.x), __float_as_int(mr3.y));
    }
    s.pm = __fadd2_rn(s.pm, mr);
    s.ax = __ffma2_rn(mr3, dx, s.ax);
    s.ay = __ffma2_rn(mr3, dy, s.ay);
    s.az = __ffma2_rn(mr3, dz, s.az);
    s.jx = __ffma2_rn(mr3, __ffma2_rn(a3, dx, dvx), s.jx);
    s.jy = __ffma2_rn(mr3, __ffma2_rn(a3, dy, dvy), s.jy);
    s.jz = __ffma2_rn(mr3, __ffma2_rn(a3, dz, dvz), s.jz);
    if (r2nn.x < s.nr2) {
        s.nr2 = r2nn.x;
        s.nj = jg0;
    }
    if (r2nn.y < s.nr2) {
        s.nr2 = r2nn.y;
        s.nj = jg0 + 1;
    }
    if (NB) {
        const bool hit0 = CHK && self0 ? (p.include_self && s.h2 > 0.f) : (r2n.x < s.h2);
        const bool hit1 = CHK && self1 ? (p.include_self && s.h2 > 0.f) : (r2n.y < s.h2);
        if (hit0) nb_push(p, s.i, jg0);
        if (hit1) nb_push(p, s.i, jg0 + 1);
    }
}

__device__ __forceinline__ void fold(StateMixedP &s) {
    s.Ax += (double)s.ax.x; s.Ax += (double)s.ax.y;
    s.Ay += (double)s.ay.x; s.Ay += (double)s.ay.y;
    s.Az += (double)s.az.x; s.Az += (double)s.az.y;
    s.Jx += (double)s.jx.x; s.Jx += (double)s.jx.y;
    s.Jy += (double)s.jy.x; s.Jy += (double)s.jy.y;
    s.Jz += (double)s.jz.x; s.Jz += (double)s.jz.y;
    s.Pt -= 4.0 * (double)s.pm.x; s.Pt -= 4.0 * (double)s.pm.y;  // pm sums m/(4r)
    s.ax = s.ay = s.az = s.jx = s.jy = s.jz = s.pm = make_float2(0.f, 0.f);
}

__device__ __forceinline__ void fold_pot(StateMixedP &s) {
    s.Pt -= 4.0 * (double)s.pm.x; s.Pt -= 4.0 * (double)s.pm.y;  // pm sums m/(4r)
    s.pm = make_float2(0.f, 0.f);
}

template <bool PO>
__device__ __forceinline__ void fold_any(StateMixedP &s) {
    if constexpr (PO)
        fold_pot(s);
    else
        fold(s);
}

__device__ __forceinline__ void fold(StateMixedBase &s) {
    s.Ax += (double)s.ax;
    s.Ay += (double)s.ay;
    s.Az += (double)s.az;
    s.Jx += (double)s.jx;
    s.Jy += (double)s.jy;
    s.Jz += (double)s.jz;
    s.Pt += (double)s.pt;
    s.ax = s.ay = s.az = s.jx = s.jy = s.jz = s.pt = 0.f;
}

// Variant bits of the mixed kernels: 2 = inner j-loop of the scalar layout
// unrolled by 4 (else 2): 1.3% faster.  (The paired layout's loop is
// unrolled by 16 with the indicators on, by 4 otherwise.)
constexpr int kVarUnroll4 = 2;
// 4 = GRAPE-4 pipeline (FP64 kernel only; see the file header).
constexpr int kVarG4 = 4;
// 8 = potential only (paired mixed and FP64 layouts): the energy sweeps.
constexpr int kVarPot = 8;
// 16 = paired mixed layout: also track the refinement's error indicators
// (the largest single acc and jerk terms: one FP32x2 multiply and two
// three-input integer maxima per pair of j).
constexpr int kVarStats = 16;

// Consume one shared-memory tile: this thread's j are kbase + m*JL.
template <int K, int R, int JL, bool CHK, bool NB, bool IDENT, int V>
__device__ __forceinline__ void consume_tile(typename StateOf<K>::type (&st)[R],
                                             const typename Traits<K>::JRec *S, int kbase,
                                             int per, int tb, const ForceParams &p) {
    if constexpr (K == kKernMixedP) {
        constexpr bool PO = (V & kVarPot) != 0;
        constexpr bool ST = (V & kVarStats) != 0;
        const float2 eps2 = dup((float)p.eps2);
        constexpr int kFlushPairs = kFlush / 2;
        if constexpr (kFlushPairs <= 2) {
            // Short folds: every one or two pair records go into FP64.
#pragma unroll 4
            for (int m = 0; m < per; m += kFlushPairs) {
#pragma unroll
                for (int u = 0; u < kFlushPairs; ++u) {
                    if (u == 0 || m + u < per) {
                        const int k = kbase + (m + u) * JL;
                        const JPairMixed J = S[k];
#pragma unroll
                        for (int r = 0; r < R; ++r)
                            interact_pair<CHK, NB, IDENT, PO, ST>(st[r], J, tb + 2 * k, eps2, p);
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r) fold_any<PO>(st[r]);
            }
            return;
        }
        // The single-call kernels (error indicators on) unroll by 16
        // (measured against 2, 4, 8 and 32 on the N = 262144 sweep: 97.6 ms
        // at 4, 95.1 at 16; 32 spills); the batched and resident kernels,
        // which hold three lane shapes in one body, by 4 (at 16 they spill).
        for (int m0 = 0; m0 < per; m0 += kFlushPairs) {
            const int m1 = min(m0 + kFlushPairs, per);
            if constexpr (ST) {
#pragma unroll 16
                for (int m = m0; m < m1; ++m) {
                    const int k = kbase + m * JL;
                    const JPairMixed J = S[k];
#pragma unroll
                    for (int r = 0; r < R; ++r) interact_pair<CHK, NB, IDENT, PO, ST>(st[r], J, tb + 2 * k, eps2, p);
                }
            } else {
#pragma unroll 4
                for (int m = m0; m < m1; ++m) {
                    const int k = kbase + m * JL;
                    const JPairMixed J = S[k];
#pragma unroll
                    for (int r = 0; r < R; ++r) interact_pair<CHK, NB, IDENT, PO, ST>(st[r], J, tb + 2 * k, eps2, p);
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) fold_any<PO>(st[r]);
        }
    } else if constexpr (K == kKernF64) {
        const double eps2 = p.eps2;
#pragma unroll 2
        for (int m = 0; m < per; ++m) {
            const int k = kbase + m * JL;
            const double4 pos = S[k].pos;
            const double4 vel = S[k].vel;
#pragma unroll
            for (int r = 0; r < R; ++r)
                interact<CHK, NB, IDENT, (V & kVarG4) != 0, (V & kVarPot) != 0>(st[r], pos, vel, tb + k, eps2, p);
        }
    } else {
        const float eps2 = (float)p.eps2;
        for (int m0 = 0; m0 < per; m0 += kFlush) {
            const int m1 = min(m0 + kFlush, per);
            if (V & kVarUnroll4) {
#pragma unroll 4
                for (int m = m0; m < m1; ++m) {
                    const int k = kbase + m * JL;
                    const auto J = S[k];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        JMixed d;
                        diff(st[r], J, d);
                        interact_mixed<CHK, NB, IDENT>(st[r], d, tb + k, eps2, p);
                    }
                }
            } else {
#pragma unroll 2
                for (int m = m0; m < m1; ++m) {
                    const int k = kbase + m * JL;
                    const auto J = S[k];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        JMixed d;
                        diff(st[r], J, d);
                        interact_mixed<CHK, NB, IDENT>(st[r], d, tb + k, eps2, p);
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) fold(st[r]);
        }
    }
}

__device__ __forceinline__ void take_min(double &r2, int &j, double o_r2, int o_j) {
    if (o_r2 < r2 || (o_r2 == r2 && (unsigned)o_j < (unsigned)j)) {
        r2 = o_r2;
        j = o_j;
    }
}

__device__ __forceinline__ void to_partial(const StateMixedBase &s, Partial &q) {
    q.acc[0] = s.Ax; q.acc[1] = s.Ay; q.acc[2] = s.Az;
    q.jerk[0] = s.Jx; q.jerk[1] = s.Jy; q.jerk[2] = s.Jz;
    q.pot = s.Pt;
    q.nn_r2 = (double)s.nr2;
    q.nn_j = s.nj;
    q.qa = q.qj = 0.f;
}
__device__ __forceinline__ void to_partial(const StateMixedP &s, Partial &q) {
    q.acc[0] = s.Ax; q.acc[1] = s.Ay; q.acc[2] = s.Az;
    q.jerk[0] = s.Jx; q.jerk[1] = s.Jy; q.jerk[2] = s.Jz;
    q.pot = s.Pt;
    q.nn_r2 = (double)s.nr2;
    q.nn_j = s.nj;
    q.qa = -2.f * __uint_as_float(s.qa);  // max m / r^2
    q.qj = __int_as_float(s.qj);          // max m / r^3
}
__device__ __forceinline__ void to_partial(const StateF64 &s, Partial &q) {
    q.acc[0] = s.Ax; q.acc[1] = s.Ay; q.acc[2] = s.Az;
    q.jerk[0] = s.Jx; q.jerk[1] = s.Jy; q.jerk[2] = s.Jz;
    q.pot = s.Pt;
    q.nn_r2 = s.nr2;
    q.nn_j = s.nj;
    q.qa = q.qj = 0.f;
}

__device__ __forceinline__ void add_partial(Partial &a, const Partial &b) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        a.acc[c] += b.acc[c];
        a.jerk[c] += b.jerk[c];
    }
    a.pot += b.pot;
    take_min(a.nn_r2, a.nn_j, b.nn_r2, b.nn_j);
    a.qa = fmaxf(a.qa, b.qa);
    a.qj = fmaxf(a.qj, b.qj);
}

// Sum over the lanes of a warp that share an i (lane bits >= log2(IL)).
template <int IL>
__device__ __forceinline__ void warp_reduce(Partial &q) {
#pragma unroll
    for (int off = IL; off < 32; off <<= 1) {
        Partial o;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            o.acc[c] = __shfl_xor_sync(0xffffffffu, q.acc[c], off);
            o.jerk[c] = __shfl_xor_sync(0xffffffffu, q.jerk[c], off);
        }
        o.pot = __shfl_xor_sync(0xffffffffu, q.pot, off);
        o.nn_r2 = __shfl_xor_sync(0xffffffffu, q.nn_r2, off);
        o.nn_j = __shfl_xor_sync(0xffffffffu, q.nn_j, off);
        o.qa = __shfl_xor_sync(0xffffffffu, q.qa, off);
        o.qj = __shfl_xor_sync(0xffffffffu, q.qj, off);
        add_partial(q, o);
    }
}

// Partial written by another CTA of the same launch: read around L1.
__device__ __forceinline__ Partial load_partial_cg(const Partial *src) {
    Partial a;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        a.acc[c] = __ldcg(&src->acc[c]);
        a.jerk[c] = __ldcg(&src->jerk[c]);
    }
    a.pot = __ldcg(&src->pot);
    a.nn_r2 = __ldcg(&src->nn_r2);
    a.nn_j = __ldcg(&src->nn_j);
    a.qa = __ldcg(&src->qa);
    a.qj = __ldcg(&src->qj);
    return a;
}

// MAPPED: honour p.out_map (only the FP64 layout's kernels, which run the
// refinement's pass, and the generic reduction kernels compile it in: in
// the paired mixed batch kernel it cost 100 bytes of spills).
template <bool MAPPED = true>
__device__ __forceinline__ void write_final(const ForceParams &p, int i, const Partial &q) {
    const size_t o = MAPPED && p.out_map ? (size_t)p.out_map[i] : (size_t)i;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        p.out_acc[3 * o + c] = q.acc[c];
        p.out_jerk[3 * o + c] = q.jerk[c];
    }
    p.out_pot[o] = q.pot;
    p.out_nn[o] = (q.nn_j < 0 || q.nn_j >= p.nj) ? 0 : q.nn_j;
    if (p.out_q) {
        p.out_q[2 * o] = q.qa;
        p.out_q[2 * o + 1] = q.qj;
    }
}

// Resident CTAs per SM the register budget is sized for (3 for the paired
// kernel measured 1.7% slower: 80 registers with spills).
template <int K, int R> struct MinBlocks {
    static constexpr int value = R >= 4 ? 1 : 2;
};

// One task: the i-tile `itile_idx` of item p against its j-split `split`.
// Shared memory holds the two mbarriers (initialised by the caller) and the
// tile ring; `gt` counts the tiles this CTA consumed before (it sets the
// ring stage and the mbarrier phase, so a persistent CTA can run many
// tasks back to back).
template <int K, int IL, int R, bool NB, bool IDENT, int V>
__device__ __forceinline__ bool process_task(const ForceParams &p, int itile_idx, int split, unsigned char *smem,
                                             int &gt) {
    using Tr = Traits<K>;
    using JRec = typename Tr::JRec;
    using State = typename StateOf<K>::type;
    constexpr int T = Tr::T;     // j per tile
    constexpr int U = Tr::U;     // records per tile
    constexpr int JPU = Tr::JPU; // j per record
    constexpr int JL = 32 / IL;
    constexpr unsigned kTileBytes = U * sizeof(JRec);

    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);          // [2], never reused
    JRec *tiles = reinterpret_cast<JRec *>(smem + 128);           // [2][U]
    Partial *red = reinterpret_cast<Partial *>(smem + 128);       // epilogue reuse

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int NW = blockDim.x >> 5;
    const int H = p.H;
    const int G = NW / H;
    const int g = warp % G, h = warp / G;
    const int il = lane % IL, jl = lane / IL;
    const int itile = G * IL * R;
    const int islot = g * IL * R + il;  // slot of r = 0 inside the i-tile
    const int i0 = itile_idx * itile + islot;

    State st[R];
    bool range_ok = true;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = i0 + r * IL;
        const bool valid = i < p.ni;
        load_i(st[r], p.irec[valid ? i : p.ni - 1], p, range_ok);
        if constexpr (K == kKernF64 && (V & kVarG4) != 0) st[r].eps2 = p.ieps2[valid ? i : p.ni - 1];
        st[r].i = i;
        if (!valid) st[r].h2 = 0;
    }
    if (!range_ok) atomicOr(p.status, ST_RANGE);

    const int jb = split * p.jper;
    const int je = min(jb + p.jper, p.nj_pad);
    const int ntiles = max(0, (je - jb) / T);
    const JRec *jrec = reinterpret_cast<const JRec *>(p.jrec);
    const int g0 = gt;

    // The previous task's epilogue may still read the tile area.
    __syncthreads();
    if (threadIdx.x == 0 && ntiles > 0) {
        const int b = g0 & 1;
        mbar_arrive_expect_tx(&bars[b], kTileBytes);
        bulk_g2s(tiles + b * U, jrec + jb / JPU, kTileBytes, &bars[b]);
    }

    const int per = U / (H * JL);
    const int kbase = h * (U / H) + jl;
    bool ok = true;
    int t = 0;
    for (; t < ntiles; ++t) {
        const int gg = g0 + t;
        const int b = gg & 1;
        if (threadIdx.x == 0 && t + 1 < ntiles) {
            mbar_arrive_expect_tx(&bars[b ^ 1], kTileBytes);
            bulk_g2s(tiles + (b ^ 1) * U, jrec + (jb + (t + 1) * T) / JPU, kTileBytes, &bars[b ^ 1]);
        }
        const bool arrived = mbar_wait_bounded(&bars[b], (gg >> 1) & 1, kWaitLimitNs);
        const JRec *S = tiles + b * U;
        const int tb = jb + t * T;
        bool chk = true;
        if (IDENT) {
            bool mine = false;
#pragma unroll
            for (int r = 0; r < R; ++r) mine |= (unsigned)(st[r].idx - tb) < (unsigned)T;
            chk = __any_sync(0xffffffffu, mine);
        }
        if (chk)
            consume_tile<K, R, JL, true, NB, IDENT, V>(st, S, kbase, per, tb, p);
        else
            consume_tile<K, R, JL, false, NB, IDENT, V>(st, S, kbase, per, tb, p);
        // The barrier that frees the tile buffer for the next copy also makes
        // a timed-out wait (on any thread) the whole CTA's decision.
        if (__syncthreads_or(!arrived)) {
            ok = false;
            break;
        }
    }
    gt = g0 + ntiles;
    if (!ok) {
        // A tile copy did not arrive within its bound: no further copy is
        // issued and the remaining tiles are skipped.  Before the epilogue
        // reuses the tile area, wait (bounded again) for this CTA's copies
        // still in flight -- tile t and, when it was issued, tile t + 1.
        if (threadIdx.x == 0) {
            const int gg = g0 + t;
            mbar_wait_bounded(&bars[gg & 1], (gg >> 1) & 1, kWaitLimitNs);
            if (t + 1 < ntiles) mbar_wait_bounded(&bars[(gg + 1) & 1], ((gg + 1) >> 1) & 1, kWaitLimitNs);
            atomicOr(p.status, ST_TMA_TIMEOUT);
        }
        __syncthreads();
    }

    // ---- epilogue: lanes -> warps -> (output | split partial)
    Partial q[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        to_partial(st[r], q[r]);
        if (JL > 1) warp_reduce<IL>(q[r]);
    }
    if (H > 1) {
        if (jl == 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) red[h * itile + islot + r * IL] = q[r];
        }
        __syncthreads();
        if (h == 0 && jl == 0) {
            for (int hh = 1; hh < H; ++hh) {
#pragma unroll
                for (int r = 0; r < R; ++r) add_partial(q[r], red[hh * itile + islot + r * IL]);
            }
        }
    }
    if (h == 0 && jl == 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = i0 + r * IL;
            if (i >= p.ni) continue;
            if (p.nsplit == 1 && !p.keep_partials)
                write_final<K == kKernF64>(p, i, q[r]);
            else
                p.part[(size_t)split * p.ni + i] = q[r];
        }
    }
    if (p.nsplit > 1 && p.tile_counter && !p.keep_partials) {
        // Last CTA of this i-tile folds the splits (threadfence reduction).
        __shared__ int s_last;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_last = atomicAdd(&p.tile_counter[itile_idx], 1) == p.nsplit - 1;
        __syncthreads();
        if (s_last) {
            __threadfence();
            const int ib = itile_idx * itile;
            for (int k = threadIdx.x; k < itile; k += blockDim.x) {
                const int i = ib + k;
                if (i >= p.ni) continue;
                Partial a = load_partial_cg(p.part + i);
                // Split order kept; four loads in flight per step (the fold is
                // latency-bound when there are many splits).
                int sp = 1;
                for (; sp + 4 <= p.nsplit; sp += 4) {
                    Partial b[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) b[u] = load_partial_cg(p.part + (size_t)(sp + u) * p.ni + i);
#pragma unroll
                    for (int u = 0; u < 4; ++u) add_partial(a, b[u]);
                }
                for (; sp < p.nsplit; ++sp) add_partial(a, load_partial_cg(p.part + (size_t)sp * p.ni + i));
                write_final<K == kKernF64>(p, i, a);
            }
            if (threadIdx.x == 0) p.tile_counter[itile_idx] = 0;
        }
    }
    return ok;
}

__device__ __forceinline__ void init_bars(unsigned char *smem) {
    if (threadIdx.x == 0) {
        uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
}

}  // namespace g6
