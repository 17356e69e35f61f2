// force.cu -- the i-block x j-particle direct-summation kernel.
//
// Pair terms are those of the reference's accumulate_acc_and_jerk
// (src/node/dyn/hdyn/evolve/hdyn_ev.C:2019-2036): with dr = x_j - x_i,
// dv = v_j - v_i, r2 = dr.dr + eps2,
//     pot -= m/r,  acc += m dr / r^3,  jerk += m/r^3 (dv - 3 (dr.dv)/r2 dr),
// self excluded by index; the nearest neighbour is the first address with
// the smallest dr.dr (no softening; hdyn_inline.C:34-77).
//
// Work decomposition (one launch):
//   gridDim.x  i-tiles;  gridDim.y  j-splits (contiguous address ranges,
//              whole tiles; their partial sums are reduced in split order by
//              reduce_partials_kernel, so the result is deterministic);
//   CTA        NW warps = G i-groups x H j-subranges;
//   warp       IL i-lanes x JL = 32/IL j-lanes; each thread owns R i's
//              (register blocking: each j read from shared memory feeds R
//              pair evaluations).
// j-tiles of T records move global -> shared by one bulk copy (TMA,
// cp.async.bulk + mbarrier) per tile, double-buffered: the copy of tile t+1
// is in flight while tile t is consumed.  Partial sums over the JL j-lanes
// are combined with warp shuffles (xor butterfly, identical on every lane),
// then over the H warps through shared memory.
//
// Mixed mode pair arithmetic is FP32 (exact position differences from the
// fixed-point split, Newton-refined rsqrt.approx); each thread sums up to
// kFlush pair terms in FP32 and then folds them into FP64 totals.  FP64 mode
// does the pair arithmetic and the sums in FP64.
#include <cfloat>
#include "common.cuh"
#include "kernels.h"

namespace g6 {

constexpr uint64_t kWaitLimitNs = 1000000000ull;  // 1 s per tile wait
constexpr int kFlush = 64;                        // FP32 terms per FP64 fold
constexpr int kMaxWarps = 8;

template <int MODE> struct Traits;
template <> struct Traits<kModeMixed> {
    using JRec = JRecMixed;
    static constexpr int T = 256;
};
template <> struct Traits<kModeF64> {
    using JRec = JRecF64;
    static constexpr int T = 128;
};

int tile_size(int mode) { return mode == kModeMixed ? Traits<kModeMixed>::T : Traits<kModeF64>::T; }

// ----------------------------------------------------------------------------
// Per-i register state.

struct StateMixed {
    float xh, yh, zh, xl, yl, zl, vx, vy, vz, h2;
    float ax, ay, az, jx, jy, jz, pt;   // FP32 sums since the last fold
    double Ax, Ay, Az, Jx, Jy, Jz, Pt;  // FP64 totals
    float nr2;
    int nj, idx, i;
};

struct StateF64 {
    double x, y, z, vx, vy, vz, h2;
    double Ax, Ay, Az, Jx, Jy, Jz, Pt;
    double nr2;
    int nj, idx, i;
};

template <int MODE> struct StateOf;
template <> struct StateOf<kModeMixed> { using type = StateMixed; };
template <> struct StateOf<kModeF64> { using type = StateF64; };

__device__ __forceinline__ void nb_push(const ForceParams &p, int i, int j) {
    int k = atomicAdd(&p.nb_count[i], 1);
    if (k < p.nb_cap) p.nb_list[(size_t)i * p.nb_cap + k] = j;
}

__device__ __forceinline__ void load_i(StateMixed &s, const IRec &q, const ForceParams &p, bool &range_ok) {
    range_ok &= to_fixed_split(q.x[0], p.fs, s.xh, s.xl);
    range_ok &= to_fixed_split(q.x[1], p.fs, s.yh, s.yl);
    range_ok &= to_fixed_split(q.x[2], p.fs, s.zh, s.zl);
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

// One pair evaluation.  CHK: the tile may hold i itself (compare ids).
template <bool CHK, bool NB, bool IDENT>
__device__ __forceinline__ void interact(StateMixed &s, const float4 &hi, const float4 &lo,
                                         const float4 &ve, int jg, float eps2,
                                         const ForceParams &p) {
    const float dx = (hi.x - s.xh) + (lo.x - s.xl);
    const float dy = (hi.y - s.yh) + (lo.y - s.yl);
    const float dz = (hi.z - s.zh) + (lo.z - s.zl);
    const float dvx = ve.x - s.vx;
    const float dvy = ve.y - s.vy;
    const float dvz = ve.z - s.vz;
    const float r2n = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float rv = fmaf(dz, dvz, fmaf(dy, dvy, dx * dvx));
    float r2 = r2n + eps2;
    float mj = hi.w;
    float r2nn = r2n;
    bool self = false;
    if (CHK) {
        self = IDENT ? (jg == s.idx) : (__float_as_int(lo.w) == s.idx);
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
    s.ax = fmaf(mr3, dx, s.ax);
    s.ay = fmaf(mr3, dy, s.ay);
    s.az = fmaf(mr3, dz, s.az);
    s.jx = fmaf(mr3, fmaf(a3, dx, dvx), s.jx);
    s.jy = fmaf(mr3, fmaf(a3, dy, dvy), s.jy);
    s.jz = fmaf(mr3, fmaf(a3, dz, dvz), s.jz);
    if (r2nn < s.nr2) {
        s.nr2 = r2nn;
        s.nj = jg;
    }
    if (NB) {
        bool hit = CHK && self ? (p.include_self && s.h2 > 0.f) : (r2n < s.h2);
        if (hit) nb_push(p, s.i, jg);
    }
}

template <bool CHK, bool NB, bool IDENT>
__device__ __forceinline__ void interact(StateF64 &s, const double4 &pos, const double4 &vel,
                                         int jg, double eps2, const ForceParams &p) {
    const double dx = pos.x - s.x;
    const double dy = pos.y - s.y;
    const double dz = pos.z - s.z;
    const double dvx = vel.x - s.vx;
    const double dvy = vel.y - s.vy;
    const double dvz = vel.z - s.vz;
    const double r2n = dx * dx + dy * dy + dz * dz;
    const double rv = dx * dvx + dy * dvy + dz * dvz;
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

__device__ __forceinline__ void fold(StateMixed &s) {
    s.Ax += (double)s.ax;
    s.Ay += (double)s.ay;
    s.Az += (double)s.az;
    s.Jx += (double)s.jx;
    s.Jy += (double)s.jy;
    s.Jz += (double)s.jz;
    s.Pt += (double)s.pt;
    s.ax = s.ay = s.az = s.jx = s.jy = s.jz = s.pt = 0.f;
}
__device__ __forceinline__ void fold(StateF64 &) {}

// Consume one shared-memory tile: this thread's j are kbase + m*JL.
template <int MODE, int R, int JL, bool CHK, bool NB, bool IDENT>
__device__ __forceinline__ void consume_tile(typename StateOf<MODE>::type (&st)[R],
                                             const typename Traits<MODE>::JRec *S, int kbase,
                                             int per, int tb, const ForceParams &p) {
    if constexpr (MODE == kModeMixed) {
        const float eps2 = (float)p.eps2;
        for (int m0 = 0; m0 < per; m0 += kFlush) {
            const int m1 = min(m0 + kFlush, per);
#pragma unroll 2
            for (int m = m0; m < m1; ++m) {
                const int k = kbase + m * JL;
                const float4 hi = S[k].hi;
                const float4 lo = S[k].lo;
                const float4 ve = S[k].vel;
#pragma unroll
                for (int r = 0; r < R; ++r) interact<CHK, NB, IDENT>(st[r], hi, lo, ve, tb + k, eps2, p);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) fold(st[r]);
        }
    } else {
        const double eps2 = p.eps2;
#pragma unroll 2
        for (int m = 0; m < per; ++m) {
            const int k = kbase + m * JL;
            const double4 pos = S[k].pos;
            const double4 vel = S[k].vel;
#pragma unroll
            for (int r = 0; r < R; ++r) interact<CHK, NB, IDENT>(st[r], pos, vel, tb + k, eps2, p);
        }
    }
}

__device__ __forceinline__ void take_min(double &r2, int &j, double o_r2, int o_j) {
    if (o_r2 < r2 || (o_r2 == r2 && (unsigned)o_j < (unsigned)j)) {
        r2 = o_r2;
        j = o_j;
    }
}

__device__ __forceinline__ void to_partial(const StateMixed &s, Partial &q) {
    q.acc[0] = s.Ax; q.acc[1] = s.Ay; q.acc[2] = s.Az;
    q.jerk[0] = s.Jx; q.jerk[1] = s.Jy; q.jerk[2] = s.Jz;
    q.pot = s.Pt;
    q.nn_r2 = (double)s.nr2;
    q.nn_j = s.nj;
}
__device__ __forceinline__ void to_partial(const StateF64 &s, Partial &q) {
    q.acc[0] = s.Ax; q.acc[1] = s.Ay; q.acc[2] = s.Az;
    q.jerk[0] = s.Jx; q.jerk[1] = s.Jy; q.jerk[2] = s.Jz;
    q.pot = s.Pt;
    q.nn_r2 = s.nr2;
    q.nn_j = s.nj;
}

__device__ __forceinline__ void add_partial(Partial &a, const Partial &b) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        a.acc[c] += b.acc[c];
        a.jerk[c] += b.jerk[c];
    }
    a.pot += b.pot;
    take_min(a.nn_r2, a.nn_j, b.nn_r2, b.nn_j);
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
        add_partial(q, o);
    }
}

__device__ __forceinline__ void write_final(const ForceParams &p, int i, const Partial &q) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        p.out_acc[3 * i + c] = q.acc[c];
        p.out_jerk[3 * i + c] = q.jerk[c];
    }
    p.out_pot[i] = q.pot;
    p.out_nn[i] = (q.nn_j < 0 || q.nn_j >= p.nj) ? 0 : q.nn_j;
}

template <int MODE, int IL, int R, bool NB, bool IDENT>
__global__ void __launch_bounds__(256, 2) force_kernel(const ForceParams p) {
    using Tr = Traits<MODE>;
    using JRec = typename Tr::JRec;
    using State = typename StateOf<MODE>::type;
    constexpr int T = Tr::T;
    constexpr int JL = 32 / IL;
    constexpr unsigned kTileBytes = T * sizeof(JRec);

    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);          // [2], never reused
    JRec *tiles = reinterpret_cast<JRec *>(smem + 128);           // [2][T]
    Partial *red = reinterpret_cast<Partial *>(smem + 128);       // epilogue reuse

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int NW = blockDim.x >> 5;
    const int H = p.H;
    const int G = NW / H;
    const int g = warp % G, h = warp / G;
    const int il = lane % IL, jl = lane / IL;
    const int itile = G * IL * R;
    const int islot = g * IL * R + il;  // slot of r = 0 inside the i-tile
    const int i0 = blockIdx.x * itile + islot;

    State st[R];
    bool range_ok = true;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = i0 + r * IL;
        const bool valid = i < p.ni;
        load_i(st[r], p.irec[valid ? i : p.ni - 1], p, range_ok);
        st[r].i = i;
        if (!valid) st[r].h2 = 0;
    }
    if (!range_ok) atomicOr(p.status, ST_RANGE);

    const int s = blockIdx.y;
    const int jb = s * p.jper;
    const int je = min(jb + p.jper, p.nj_pad);
    const int ntiles = (je - jb) / T;
    const JRec *jrec = reinterpret_cast<const JRec *>(p.jrec);

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && ntiles > 0) {
        mbar_arrive_expect_tx(&bars[0], kTileBytes);
        bulk_g2s(tiles, jrec + jb, kTileBytes, &bars[0]);
    }

    const int per = T / (H * JL);
    const int kbase = h * (T / H) + jl;
    bool ok = true;
    for (int t = 0; t < ntiles; ++t) {
        const int b = t & 1;
        if (threadIdx.x == 0 && t + 1 < ntiles) {
            mbar_arrive_expect_tx(&bars[b ^ 1], kTileBytes);
            bulk_g2s(tiles + (b ^ 1) * T, jrec + jb + (t + 1) * T, kTileBytes, &bars[b ^ 1]);
        }
        if (ok) ok = mbar_wait_bounded(&bars[b], (t >> 1) & 1, kWaitLimitNs);
        const JRec *S = tiles + b * T;
        const int tb = jb + t * T;
        bool chk = true;
        if (IDENT) {
            bool mine = false;
#pragma unroll
            for (int r = 0; r < R; ++r) mine |= (unsigned)(st[r].idx - tb) < (unsigned)T;
            chk = __any_sync(0xffffffffu, mine);
        }
        if (chk)
            consume_tile<MODE, R, JL, true, NB, IDENT>(st, S, kbase, per, tb, p);
        else
            consume_tile<MODE, R, JL, false, NB, IDENT>(st, S, kbase, per, tb, p);
        __syncthreads();
    }
    if (!ok) atomicOr(p.status, ST_TMA_TIMEOUT);

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
            if (p.nsplit == 1)
                write_final(p, i, q[r]);
            else
                p.part[(size_t)s * p.ni + i] = q[r];
        }
    }
}

__global__ void reduce_partials_kernel(const ForceParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.ni) return;
    Partial a = p.part[i];
    for (int s = 1; s < p.nsplit; ++s) add_partial(a, p.part[(size_t)s * p.ni + i]);
    write_final(p, i, a);
}

// ----------------------------------------------------------------------------
// Host side: kernel selection and launch geometry.

using KernelFn = void (*)(const ForceParams);

template <int MODE, int IL, int R>
static KernelFn pick3(bool nb, bool ident) {
    if (nb) return ident ? force_kernel<MODE, IL, R, true, true> : force_kernel<MODE, IL, R, true, false>;
    return ident ? force_kernel<MODE, IL, R, false, true> : force_kernel<MODE, IL, R, false, false>;
}

template <int MODE>
static KernelFn pick2(int il, int r, bool nb, bool ident) {
    if (il == 32) return r == 2 ? pick3<MODE, 32, 2>(nb, ident) : pick3<MODE, 32, 1>(nb, ident);
    if (il == 8) return pick3<MODE, 8, 1>(nb, ident);
    return pick3<MODE, 1, 1>(nb, ident);
}

static KernelFn pick(int mode, int il, int r, bool nb, bool ident) {
    return mode == kModeMixed ? pick2<kModeMixed>(il, r, nb, ident) : pick2<kModeF64>(il, r, nb, ident);
}

static size_t smem_bytes(int mode, const ForceConfig &c) {
    size_t rec = mode == kModeMixed ? sizeof(JRecMixed) : sizeof(JRecF64);
    size_t tiles = 2 * (size_t)tile_size(mode) * rec;
    size_t itile = (size_t)(c.warps / c.H) * c.il * c.r;
    size_t red = c.H > 1 ? (size_t)c.H * itile * sizeof(Partial) : 0;
    return 128 + (tiles > red ? tiles : red);
}

size_t partial_bytes(const ForceConfig &cfg, int ni) {
    return cfg.nsplit > 1 ? (size_t)cfg.nsplit * ni * sizeof(Partial) : 0;
}

ForceConfig choose_config(int mode, int ni, int nj_pad, int num_sms, bool nb) {
    (void)nb;
    ForceConfig c;
    c.warps = kMaxWarps;
    c.il = ni >= 32 ? 32 : (ni > 1 ? 8 : 1);
    if (c.il == 8 && ni > 8) c.il = 32;
    c.r = (mode == kModeMixed && c.il == 32 && ni >= 8192) ? 2 : 1;
    // i-groups per CTA: as many warps on distinct i as there are i's.
    int groups_needed = (ni + c.il * c.r - 1) / (c.il * c.r);
    int G = 1;
    while (G * 2 <= c.warps && G * 2 <= groups_needed) G *= 2;
    c.H = c.warps / G;
    const int T = tile_size(mode);
    const int JL = 32 / c.il;
    while (c.H > 1 && T / (c.H * JL) < 1) c.H /= 2;  // keep >= 1 j per thread per tile
    G = c.warps / c.H;
    const int itile = G * c.il * c.r;
    const int n_itiles = (ni + itile - 1) / itile;
    const int ntiles = nj_pad / T;
    // Fill the GPU with whole waves: 2 resident CTAs per SM.
    const int slots = 2 * num_sms;
    int best_split = 1;
    double best_eff = -1;
    for (int sp = 1; sp <= ntiles && sp <= 4096; ++sp) {
        const int per_split_tiles = (ntiles + sp - 1) / sp;
        const int real_split = (ntiles + per_split_tiles - 1) / per_split_tiles;
        if (real_split != sp) continue;
        const long long ctas = (long long)n_itiles * sp;
        const long long waves = (ctas + slots - 1) / slots;
        double eff = (double)ctas / (double)(waves * slots);
        // Penalise tiny per-CTA work (tile pipeline start-up, reduction).
        if (per_split_tiles < 4 && sp > 1) eff *= 0.5;
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best_split = sp;
        }
        if (ctas >= 8LL * slots) break;
    }
    c.nsplit = best_split;
    return c;
}

cudaError_t launch_force(cudaStream_t s, int mode, const ForceConfig &cfg, ForceParams p,
                         bool ident, bool nb) {
    const int T = tile_size(mode);
    const int ntiles = p.nj_pad / T;
    if (p.ni <= 0) return cudaSuccess;
    if (ntiles <= 0) {
        p.jper = T;
        p.nsplit = 1;
    } else {
        const int per_split_tiles = (ntiles + cfg.nsplit - 1) / cfg.nsplit;
        p.jper = per_split_tiles * T;
        p.nsplit = (ntiles + per_split_tiles - 1) / per_split_tiles;
    }
    p.H = cfg.H;
    const int G = cfg.warps / cfg.H;
    const int itile = G * cfg.il * cfg.r;
    dim3 grid((p.ni + itile - 1) / itile, p.nsplit);
    dim3 block(32 * cfg.warps);
    KernelFn fn = pick(mode, cfg.il, cfg.r, nb, ident);
    size_t sm = smem_bytes(mode, cfg);
    fn<<<grid, block, sm, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (p.nsplit > 1) {
        reduce_partials_kernel<<<(p.ni + 255) / 256, 256, 0, s>>>(p);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace g6
