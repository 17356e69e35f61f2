// ensemble.cu -- many independent clusters integrated together on one GPU.
//
// Each cluster is advanced with the 4th-order Hermite scheme and
// individual power-of-two block timesteps -- the scheme kira runs for its
// top-level nodes (kira_int.C:560 integrate_list; predictor
// include/_dyn_.h:265-299; corrector hdyn_ev.C:1717-1718; Aarseth-type
// timestep criterion with accuracy parameter eta, hdyn_ev.C:521+).  The
// j-state of every cluster stays in HBM.  One iteration advances EVERY
// active cluster by its own next block:
//
//   predict    all particles of active clusters to their own t_b (FP64),
//              j-records in the force kernel's layout; the block members
//              (t_i + dt_i == t_b) compacted into i-records
//   scan       each cluster's work item (a ForceParams: its j-records,
//              i-records, softening, fixed-point scale, outputs, split
//              plan), the task order, prefix sums of task and i counts
//   force      ONE persistent launch over the (cluster, i-tile, j-split)
//              work list of all clusters, the splits folded in-kernel
//   correct    Hermite corrector in FP64 + new timestep, in place; the
//              next block time t_b = min(t_i + dt_i) of every cluster
//              (members here, the others in predict), published by the
//              corrector's last CTA
//
// The first block step of a run (and the start and energy sweeps) take
// their block time and members from a schedule kernel instead (one CTA per
// cluster, address order).  The steady-state iteration is captured once as
// a CUDA graph and replayed.  For
// comparison, run_per_cluster drives the same integration through the plain
// single-cluster engine (one g6 firsthalf/lasthalf2 call per cluster per
// block, host-side prediction and correction) -- the way independent kira
// runs would share the GPU.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "common.cuh"
#include "engine.h"
#include "kernels.h"

namespace g6 {

struct EnsDev {
    int nc, ntot;
    const int *off, *n, *cid;
    const double *eps2;
    const FixedScale *fs;
    const long long *part_off;
    double *x, *v, *a, *jk, *t, *dt, *m;  // x/v/a/jk: [3][ntot]
    int *slot;
    double *tblock;
    int *count, *ntask;
    void *jrec;
    IRec *irec;
    double *acc1, *jerk1, *pot1;
    int *nn1;
    Partial *part;
    ForceParams *items;
    int *task0, *ipre, *counter;
    int *order;  // [nc] clusters in task order (scan kernel)
    unsigned long long *tnext;  // [nc] next block time being formed (bits of a non-negative double; min)
    unsigned *done;             // corrector CTAs finished (the last one publishes tnext)
    int *tcnt;  // per-particle slots of i-tile arrival counters (split reduction in the force kernel)
    unsigned *status;
    int *active;
    unsigned long long *interactions;
    double t_end, eta, eta_s, dt_max;
    int kmode;
    ForceConfig cfg;
};

__device__ __forceinline__ void predict_state(const EnsDev &d, int g, double tb, double xp[3], double vp[3]) {
    const double h = tb - d.t[g];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const double x = d.x[c * d.ntot + g], v = d.v[c * d.ntot + g];
        const double a2 = 0.5 * d.a[c * d.ntot + g], j6 = d.jk[c * d.ntot + g] * (1.0 / 6.0);
        xp[c] = x + h * (v + h * (a2 + h * j6));
        vp[c] = v + h * (2.0 * a2 + h * (3.0 * j6));
    }
}

// mode 0: next block; mode 1: every particle at its current time (start of
// the run, or an energy evaluation when all times are equal).
// One CTA of 512 threads per cluster.  Each step covers kSchedPer x 512
// particles, element k of a thread at base + k * 512 + tid (coalesced);
// all of a step's loads are issued before any of them is used, so a large
// cluster keeps enough bytes in flight (the kernel is latency-bound
// otherwise: one CTA walks up to 16384 particles).
constexpr unsigned long long kTimeInf = 0x7ff0000000000000ull;  // bits of +inf (tnext: no time yet)
constexpr int kSchedThreads = 512;
constexpr int kSchedPer = 8;

__global__ void __launch_bounds__(kSchedThreads) ens_schedule_kernel(EnsDev d, int mode) {
    constexpr int NW = kSchedThreads / 32;
    __shared__ double s_wmin[NW];
    __shared__ int s_wcnt[kSchedPer][NW];
    const int c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int n = d.n[c], o = d.off[c], span = d.off[c + 1] - o;  // span: n padded to 256
    const double *t = d.t + o, *dt = d.dt + o;
    double tmin = DBL_MAX;
    if (mode == 0) {
        for (int base = 0; base < n; base += kSchedPer * kSchedThreads) {
            double tn[kSchedPer];
#pragma unroll
            for (int k = 0; k < kSchedPer; ++k) {
                const int i = base + k * kSchedThreads + tid;
                tn[k] = i < n ? t[i] + dt[i] : DBL_MAX;
            }
#pragma unroll
            for (int k = 0; k < kSchedPer; ++k) tmin = fmin(tmin, tn[k]);
        }
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) tmin = fmin(tmin, __shfl_xor_sync(0xffffffffu, tmin, k));
    if (lane == 0) s_wmin[w] = tmin;
    __syncthreads();
    for (int k = 0; k < NW; ++k) tmin = fmin(tmin, s_wmin[k]);
    const double tb = mode == 0 ? tmin : (n > 0 ? d.t[o] : 0.0);
    const bool active = n > 0 && (mode != 0 || tb <= d.t_end);
    // Ordered compaction of the block members: slot = members before this
    // particle in address order.
    int running = 0;
    for (int base = 0; base < span; base += kSchedPer * kSchedThreads) {
        double tn[kSchedPer];
#pragma unroll
        for (int k = 0; k < kSchedPer; ++k) {
            const int i = base + k * kSchedThreads + tid;
            tn[k] = i < n ? t[i] + dt[i] : DBL_MAX;
        }
        unsigned bal[kSchedPer];
#pragma unroll
        for (int k = 0; k < kSchedPer; ++k) {
            bal[k] = __ballot_sync(0xffffffffu, active && (mode != 0 ? base + k * kSchedThreads + tid < n : tn[k] == tb));
            if (lane == 0) s_wcnt[k][w] = __popc(bal[k]);
        }
        __syncthreads();
        int before = running;  // members of the earlier sub-steps and warps
#pragma unroll
        for (int k = 0; k < kSchedPer; ++k) {
            int woff = 0, tot = 0;
            for (int q = 0; q < NW; ++q) {
                const int v = s_wcnt[k][q];
                woff += q < w ? v : 0;
                tot += v;
            }
            const int i = base + k * kSchedThreads + tid;
            if (i < span)
                d.slot[o + i] = (bal[k] >> lane) & 1u ? before + woff + __popc(bal[k] & ((1u << lane) - 1u)) : -1;
            before += tot;
        }
        running = before;
        __syncthreads();
    }
    if (tid == 0) {
        d.count[c] = running;
        d.tblock[c] = tb;
        d.tnext[c] = kTimeInf;
    }
}

// Work item of cluster c with ni block members.
__device__ __forceinline__ void make_item(const EnsDev &d, int c, int ni, ForceParams &p, int &nt) {
    const int o = d.off[c], n = d.n[c];
    const size_t jb = d.kmode == kKernF64 ? sizeof(JRecF64) : sizeof(JRecMixed);
    p = ForceParams{};
    p.jrec = static_cast<const char *>(d.jrec) + (size_t)o * jb;
    p.nj = n;
    p.nj_pad = (n + tile_of(d.kmode) - 1) / tile_of(d.kmode) * tile_of(d.kmode);
    p.irec = d.irec + o;
    p.ni = ni;
    p.eps2 = d.eps2[c];
    p.fs = d.fs[c];
    p.part = d.part + d.part_off[c];
    p.out_acc = d.acc1 + 3 * (size_t)o;
    p.out_jerk = d.jerk1 + 3 * (size_t)o;
    p.out_pot = d.pot1 + o;
    p.out_nn = d.nn1 + o;
    p.status = d.status;
    p.tile_counter = d.tcnt + o;  // n_itiles <= ni <= n: the last CTA of an i-tile adds its splits
    nt = 0;
    batch_plan(d.kmode, d.cfg, p, nt);
}

// Exclusive prefix sums of the clusters' task and member counts, the count
// of active clusters and the interaction total: one CTA of 1024 threads,
// each owning a contiguous run of clusters; warp-shuffle scans.
constexpr int kOrderMax = 4096;  // clusters ordered by work per task (32 KB of keys)

__global__ void __launch_bounds__(1024) ens_scan_kernel(EnsDev d) {
    __shared__ int s_t[32], s_i[32], s_a[32];
    __shared__ unsigned long long s_x[32], s_l[32];
    __shared__ long long s_key[kOrderMax];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    // Task order: clusters by descending work per task (longest tasks first,
    // so that the persistent CTAs' last tasks are short ones), ties by
    // cluster number; clusters with no task last.  Each key is computed once
    // into shared memory and ranked by counting; above kOrderMax clusters the
    // order is the cluster order.
    for (int c = tid; c < d.nc; c += 1024) {
        ForceParams p;
        int nt;
        make_item(d, c, d.count[c], p, nt);
        d.items[c] = p;
        d.ntask[c] = nt;
        if (c < kOrderMax) s_key[c] = nt > 0 ? (long long)min(batch_item_itile(d.kmode, d.cfg, p.ni), p.ni) * p.jper
                                             : -1;
    }
    __syncthreads();
    if (d.nc <= kOrderMax) {
        for (int c = tid; c < d.nc; c += 1024) {
            const long long kc = s_key[c];
            int rank = 0;
            for (int q = 0; q < d.nc; ++q) {
                const long long kq = s_key[q];
                rank += kq > kc || (kq == kc && q < c);
            }
            d.order[rank] = c;
        }
    } else {
        for (int c = tid; c < d.nc; c += 1024) d.order[c] = c;
    }
    __syncthreads();
    const int per = (d.nc + 1023) / 1024;
    const int b = min(tid * per, d.nc), e = min(b + per, d.nc);
    int lt = 0, li = 0, la = 0;
    unsigned long long lx = 0, ll = 0;
    for (int c = b; c < e; ++c) {
        const int cnt = d.count[c];
        lt += d.ntask[d.order[c]];  // tasks in the sorted order (position c)
        li += cnt;
        la += cnt > 0;
        lx += (unsigned long long)cnt * (unsigned long long)d.n[c];
        if (cnt > 0) {  // lanes the force kernel runs: whole i-tiles x padded j
            const ForceParams &p = d.items[c];
            const int it = batch_item_itile(d.kmode, d.cfg, cnt);
            ll += (unsigned long long)((cnt + it - 1) / it * it) * (unsigned long long)p.nj_pad;
        }
    }
    // inclusive warp scans of lt, li; warp sums of la, lx
    int it = lt, ii = li;
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
        const int a1 = __shfl_up_sync(0xffffffffu, it, k), a2 = __shfl_up_sync(0xffffffffu, ii, k);
        if (lane >= k) {
            it += a1;
            ii += a2;
        }
    }
    int sa = la;
    unsigned long long sx = lx, sl = ll;
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
        sa += __shfl_xor_sync(0xffffffffu, sa, k);
        sx += __shfl_xor_sync(0xffffffffu, sx, k);
        sl += __shfl_xor_sync(0xffffffffu, sl, k);
    }
    if (lane == 31) {
        s_t[w] = it;
        s_i[w] = ii;
    }
    if (lane == 0) {
        s_a[w] = sa;
        s_x[w] = sx;
        s_l[w] = sl;
    }
    __syncthreads();
    int wt = 0, wi = 0;
    for (int k = 0; k < w; ++k) {
        wt += s_t[k];
        wi += s_i[k];
    }
    int t = wt + it - lt, i2 = wi + ii - li;  // exclusive prefix of this thread's run
    for (int c = b; c < e; ++c) {
        d.task0[c] = t;  // prefix over the sorted order (position c)
        d.ipre[c] = i2;  // prefix over the clusters
        t += d.ntask[d.order[c]];
        i2 += d.count[c];
    }
    if (tid == 1023) {
        int act = 0;
        unsigned long long inter = 0, lanes = 0;
        for (int k = 0; k < 32; ++k) {
            act += s_a[k];
            inter += s_x[k];
            lanes += s_l[k];
        }
        d.task0[d.nc] = t;
        d.ipre[d.nc] = i2;
        *d.active = act;
        d.interactions[0] += inter;
        d.interactions[1] += lanes;
        *d.counter = 0;
    }
}

// Paired mixed records (one thread per pair) or FP64 records (one thread
// per particle); i-records for the block members.
//
// fused = 0: the members are those the schedule kernel listed (slot[]).
// fused = 1 (block steps after the first of a run): the block time is the
// one the previous corrector published, and the members -- t + dt equal to
// it -- are compacted here: one atomic per warp on the cluster's count, the
// warp's members in lane order after it.  The slot order then varies from
// run to run; the forces do not (each i's sums are independent of its
// slot).  Either way the non-members' t + dt go into the next block time
// (tnext, a min over bit patterns of non-negative doubles); the corrector
// adds the members' new t + dt.
//
// A warp never straddles two clusters (cluster spans are multiples of 256
// particles), so its early returns are warp-uniform and the ballots below
// see all 32 lanes.
__global__ void ens_predict_kernel(EnsDev d, int fused) {
    const int per = d.kmode == kKernMixedP ? 2 : 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int g0 = q * per;
    if (g0 >= d.ntot) return;
    const int c = d.cid[g0];
    if (c < 0) return;
    const int o = d.off[c], n = d.n[c];
    const double tb = d.tblock[c];
    if (fused ? (n == 0 || !(tb <= d.t_end)) : d.count[c] == 0) return;  // inactive: tnext stays +inf
    int sl[2] = {-1, -1};
    unsigned long long tn_min = kTimeInf;
    {
        bool mem[2] = {false, false};
        for (int u = 0; u < per; ++u) {
            const int g = g0 + u, i = g - o;
            if (i >= n) continue;
            const double tn = d.t[g] + d.dt[g];
            mem[u] = fused ? tn == tb : d.slot[g] >= 0;
            if (!mem[u]) tn_min = min(tn_min, (unsigned long long)__double_as_longlong(tn));
        }
        if (fused) {
            const unsigned lane = threadIdx.x & 31u, below = (1u << lane) - 1u;
            const unsigned b0 = __ballot_sync(0xffffffffu, mem[0]), b1 = __ballot_sync(0xffffffffu, mem[1]);
            const int tot = __popc(b0) + __popc(b1);
            int base = 0;
            if (lane == 0 && tot > 0) base = atomicAdd(&d.count[c], tot);
            base = __shfl_sync(0xffffffffu, base, 0);
            sl[0] = mem[0] ? base + __popc(b0 & below) : -1;
            sl[1] = mem[1] ? base + __popc(b0) + __popc(b1 & below) : -1;
            for (int u = 0; u < per; ++u) d.slot[g0 + u] = sl[u];
        } else {
            for (int u = 0; u < per; ++u) sl[u] = g0 + u - o < n ? d.slot[g0 + u] : -1;
        }
        for (int k = 16; k > 0; k >>= 1) tn_min = min(tn_min, __shfl_xor_sync(0xffffffffu, tn_min, k));
        if ((threadIdx.x & 31u) == 0 && tn_min != kTimeInf) atomicMin(&d.tnext[c], tn_min);
    }
    float hi[2][3], lo[2][3], vv[2][3], mm[2];
    int id[2];
    bool bad = false;
    for (int u = 0; u < per; ++u) {
        const int g = g0 + u, i = g - o;
        if (i < n) {
            double xp[3], vp[3];
            predict_state(d, g, tb, xp, vp);
            const int s = sl[u];
            if (s >= 0) {
                IRec r;
                for (int k = 0; k < 3; ++k) {
                    r.x[k] = xp[k];
                    r.v[k] = vp[k];
                }
                r.h2 = 0.0;
                r.index = i;
                r.pad = 0;
                d.irec[o + s] = r;
            }
            if (d.kmode == kKernF64) {
                JRecF64 rec;
                rec.pos = make_double4(xp[0], xp[1], xp[2], d.m[g]);
                rec.vel = make_double4(vp[0], vp[1], vp[2], (double)i);
                reinterpret_cast<JRecF64 *>(d.jrec)[g] = rec;
            } else {
                for (int k = 0; k < 3; ++k) {
                    bad |= !to_fixed_split(xp[k], d.fs[c], hi[u][k], lo[u][k]);
                    vv[u][k] = (float)vp[k];
                }
                mm[u] = (float)d.m[g];
                id[u] = i;
            }
        } else if (d.kmode == kKernF64) {
            JRecF64 rec;
            rec.pos = make_double4(kDummyPos, kDummyPos, kDummyPos, 0.0);
            rec.vel = make_double4(0.0, 0.0, 0.0, -1.0);
            reinterpret_cast<JRecF64 *>(d.jrec)[g] = rec;
        } else {
            for (int k = 0; k < 3; ++k) {
                hi[u][k] = kDummyPos;
                lo[u][k] = 0.f;
                vv[u][k] = 0.f;
            }
            mm[u] = 0.f;
            id[u] = -1;
        }
    }
    if (bad) atomicOr(d.status, ST_RANGE);
    if (d.kmode == kKernMixedP) {
        JPairMixed r;
        r.hxy = make_float4(hi[0][0], hi[1][0], hi[0][1], hi[1][1]);
        r.hzm = make_float4(hi[0][2], hi[1][2], -0.125f * mm[0], -0.125f * mm[1]);  // -m/8: see JPairMixed
        r.lxy = make_float4(lo[0][0], lo[1][0], lo[0][1], lo[1][1]);
        r.lzi = make_float4(lo[0][2], lo[1][2], __int_as_float(id[0]), __int_as_float(id[1]));
        r.vxy = make_float4(vv[0][0], vv[1][0], vv[0][1], vv[1][1]);
        r.vz = make_float4(vv[0][2], vv[1][2], 0.f, 0.f);
        reinterpret_cast<JPairMixed *>(d.jrec)[g0 / 2] = r;
    }
}

// Smallest block step: below it t + dt would no longer advance t in FP64
// for t ~ 1, so steps are floored here instead.
constexpr double kDtMin = 9.094947017729282e-13;  // 2^-40

__host__ __device__ inline double pow2_floor(double x) {
    int e;
    frexp(x, &e);  // x = f 2^e, f in [0.5, 1)
    return ldexp(1.0, e - 1);
}

// Hermite corrector (FP64) and the next block step.  mode 1 = start: take
// the forces as the initial acc/jerk and choose the first step from
// eta_s |a| / |j|.
__device__ __forceinline__ void correct_one(const EnsDev &d, int mode, int c, int o, int s, int g) {
    const double tb = d.tblock[c];
    const size_t k = (size_t)o + s;
    double a1[3], j1[3];
    for (int q = 0; q < 3; ++q) {
        a1[q] = d.acc1[3 * k + q];
        j1[q] = d.jerk1[3 * k + q];
    }
    const int N = d.ntot;
    if (mode == 1) {
        double an = 0, jn = 0;
        for (int q = 0; q < 3; ++q) {
            d.a[q * N + g] = a1[q];
            d.jk[q * N + g] = j1[q];
            an += a1[q] * a1[q];
            jn += j1[q] * j1[q];
        }
        double dt0 = (jn > 0) ? d.eta_s * sqrt(an / jn) : d.dt_max;
        dt0 = fmin(pow2_floor(fmax(dt0, kDtMin)), d.dt_max);
        d.dt[g] = dt0;
        return;
    }
    const double h = tb - d.t[g];
    double xp[3], vp[3];
    predict_state(d, g, tb, xp, vp);
    double a2e[3], a3[3];
    const double h2 = h * h, h3 = h2 * h;
    double sa1 = 0, sj1 = 0, sa2 = 0, sa3 = 0;
    for (int q = 0; q < 3; ++q) {
        const double a0 = d.a[q * N + g], j0 = d.jk[q * N + g];
        const double sn = (-6.0 * (a0 - a1[q]) - h * (4.0 * j0 + 2.0 * j1[q])) / h2;
        const double cr = (12.0 * (a0 - a1[q]) + 6.0 * h * (j0 + j1[q])) / h3;
        d.x[q * N + g] = xp[q] + h2 * h2 * (sn / 24.0 + h * cr / 120.0);
        d.v[q * N + g] = vp[q] + h3 * (sn / 6.0 + h * cr / 24.0);
        d.a[q * N + g] = a1[q];
        d.jk[q * N + g] = j1[q];
        a2e[q] = sn + h * cr;
        a3[q] = cr;
        sa1 += a1[q] * a1[q];
        sj1 += j1[q] * j1[q];
        sa2 += a2e[q] * a2e[q];
        sa3 += a3[q] * a3[q];
    }
    const double na1 = sqrt(sa1), nj1 = sqrt(sj1), na2 = sqrt(sa2), na3 = sqrt(sa3);
    const double den = nj1 * na3 + sa2;
    double dtn = den > 0 ? sqrt(d.eta * (na1 * na2 + sj1) / den) : 2.0 * h;
    dtn = pow2_floor(fmax(dtn, kDtMin));
    dtn = fmin(dtn, fmin(2.0 * h, d.dt_max));
    while (dtn > kDtMin && (fmod(tb, dtn) != 0.0 || (tb < d.t_end && tb + dtn > d.t_end))) dtn *= 0.5;
    d.t[g] = tb;
    d.dt[g] = fmax(dtn, kDtMin);
}

// Grid-stride over the block members only (ipre[nc] of them): member m is
// slot s of cluster c, particle o + irec[o + s].index.
// Each member's new t + dt goes into its cluster's tnext; the last CTA to
// finish publishes tnext as the next block time (tblock), and resets tnext
// and the member counts for the next iteration's predict kernel.
//
// Members are in cluster order, so a warp's lanes of one cluster are
// contiguous: a segmented min over the warp leaves one atomic per cluster
// per warp (the lane that heads the cluster's run).
__global__ void ens_correct_kernel(EnsDev d, int mode) {
    __shared__ bool s_last;
    const int total = d.ipre[d.nc];
    const int lane = threadIdx.x & 31;
    for (int m0 = blockIdx.x * blockDim.x; m0 < total; m0 += gridDim.x * blockDim.x) {  // block-uniform
        const int m = m0 + threadIdx.x;
        int c = -1;
        unsigned long long tn = kTimeInf;
        if (m < total) {
            int lo = 0, hi = d.nc - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (d.ipre[mid] <= m) lo = mid; else hi = mid - 1;
            }
            c = lo;
            const int s = m - d.ipre[c], o = d.off[c];
            const int g = o + d.irec[o + s].index;
            correct_one(d, mode, c, o, s, g);
            tn = (unsigned long long)__double_as_longlong(d.t[g] + d.dt[g]);
        }
#pragma unroll
        for (int k = 1; k < 32; k <<= 1) {
            const unsigned long long ot = __shfl_down_sync(0xffffffffu, tn, k);
            const int oc = __shfl_down_sync(0xffffffffu, c, k);
            if (lane + k < 32 && oc == c) tn = min(tn, ot);
        }
        const int up = __shfl_up_sync(0xffffffffu, c, 1);
        if (c >= 0 && (lane == 0 || up != c)) atomicMin(&d.tnext[c], tn);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(d.done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int c = threadIdx.x; c < d.nc; c += blockDim.x) {
        d.tblock[c] = __longlong_as_double((long long)atomicExch(&d.tnext[c], kTimeInf));
        d.count[c] = 0;
    }
    if (threadIdx.x == 0) *d.done = 0;
}

// Before a run: no step may jump over t_end, so every particle lands on it
// (t_end is a dyadic time and halving keeps t a multiple of dt).
__global__ void ens_cap_kernel(EnsDev d) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= d.ntot || d.cid[g] < 0 || g - d.off[d.cid[g]] >= d.n[d.cid[g]]) return;
    double dt = d.dt[g];
    while (dt > kDtMin && d.t[g] < d.t_end && d.t[g] + dt > d.t_end) dt *= 0.5;
    d.dt[g] = dt;
}

// Kinetic and potential energy of every cluster (FP64, fixed reduction
// order); pot1 holds the potentials of a mode-1 sweep.
__global__ void __launch_bounds__(256) ens_energy_kernel(EnsDev d, double *out) {
    __shared__ double sk[256], sp[256];
    const int c = blockIdx.x, tid = threadIdx.x;
    const int n = d.n[c], o = d.off[c], N = d.ntot;
    double ek = 0, ep = 0;
    for (int i = tid; i < n; i += 256) {
        const int g = o + i;
        const int s = d.slot[g];
        double v2 = 0;
        for (int q = 0; q < 3; ++q) v2 += d.v[q * N + g] * d.v[q * N + g];
        ek += 0.5 * d.m[g] * v2;
        if (s >= 0) ep += 0.5 * d.m[g] * d.pot1[o + s];
    }
    sk[tid] = ek;
    sp[tid] = ep;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (tid < w) {
            sk[tid] += sk[tid + w];
            sp[tid] += sp[tid + w];
        }
        __syncthreads();
    }
    if (tid == 0) {
        out[2 * c] = sk[0];
        out[2 * c + 1] = sp[0];
    }
}

// ---------------------------------------------------------------------------

struct EnsembleStats {
    double seconds = 0;
    long long interactions = 0;
    long long iterations = 0;
    long long launches = 0;
    double tuned_h = 0;
    int tuned_tasks = 0;
    long long lane_interactions = 0;  // i-lanes x j the force kernel ran (whole i-tiles, padded j)
};

class Ensemble {
  public:
    Ensemble(int nc, const int *n, const double *eps2, double eta, int mode, int device)
        : nc_(nc), n_(n, n + nc), eps2_(eps2, eps2 + nc), eta_(eta), mode_(mode), device_(device) {}
    ~Ensemble() { release(); }

    std::string err;

    int setup();
    int set_cluster(int c, const double *m, const double (*x)[3], const double (*v)[3]);
    int start();                                    // forces and first steps at t = 0
    int run_batched(double t_end, EnsembleStats *st, int tune);
    int run_per_cluster(double t_end, EnsembleStats *st);
    int energies(double *ek_ep);                    // [2 nc], all clusters at equal time
    int get_cluster(int c, double *m, double (*x)[3], double (*v)[3], double (*acc)[3], double (*jerk)[3],
                    double *t, double *dt);

  private:
    int fail(const char *what, cudaError_t e) {
        err = std::string("ensemble: ") + what + ": " + cudaGetErrorString(e);
        return -1;
    }
    void release();
    int iteration(int mode, bool fused = false);  // [schedule] -> predict -> scan -> force -> correct
    long long launches_ = 0;  // kernels launched by iteration() (not counting graph captures)
    int sync_host_state();
    int push_host_state();

    int nc_;
    std::vector<int> n_;
    std::vector<double> eps2_;
    double eta_;
    int mode_, device_;
    int kmode_ = kKernMixedP;
    int ntot_ = 0;
    long long max_iters_ = 2000000;  // run guards (G6B200_ENS_MAX_ITERS / _SECONDS)
    double max_seconds_ = 600.0;
    bool fuse_ = true;  // G6B200_ENS_FUSED=0: every block step through the schedule kernel
    int min_tiles_ = 4;  // G6B200_ENS_MIN_TILES: fewest j-tiles per task (1, 2, 4 or 8)
    std::vector<int> off_;
    std::vector<double> hm_, hx_, hv_;  // host copies of the initial state
    EnsDev d_{};
    cudaStream_t stream_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    int graph_iters_ = 0;
    int ctas_ = 0, num_sms_ = 148;
    void *blob_ = nullptr;
    std::vector<void *> allocs_;
    // host state for the per-cluster baseline: x,v,a,jk [3][ntot] + t, dt, m
    std::vector<double> sx_, sv_, sa_, sj_, st_, sdt_, sm_;
};

void Ensemble::release() {
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
    for (void *p : allocs_) cudaFree(p);
    allocs_.clear();
    if (stream_) cudaStreamDestroy(stream_);
    stream_ = nullptr;
}

#define ECHK(call, what)                              \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return fail(what, e_); \
    } while (0)

int Ensemble::setup() {
    if (const char *e = getenv("G6B200_ENS_MAX_ITERS")) max_iters_ = atoll(e);
    if (const char *e = getenv("G6B200_ENS_MAX_SECONDS")) max_seconds_ = atof(e);
    if (const char *e = getenv("G6B200_ENS_FUSED")) fuse_ = atoi(e) != 0;
    if (const char *e = getenv("G6B200_ENS_MIN_TILES")) {
        const int v = atoi(e);
        min_tiles_ = v <= 1 ? 1 : (v <= 2 ? 2 : (v <= 4 ? 4 : 8));
    }
    ECHK(cudaSetDevice(device_), "device");
    ECHK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    ECHK(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, device_), "attr");
    kmode_ = mode_ == kModeF64 ? kKernF64 : kKernMixedP;
    off_.assign(nc_ + 1, 0);
    for (int c = 0; c < nc_; ++c) off_[c + 1] = off_[c] + (n_[c] + 255) / 256 * 256;
    ntot_ = off_[nc_];
    std::vector<int> cid(ntot_, -1);
    std::vector<long long> poff(nc_);
    long long ptot = 0;
    for (int c = 0; c < nc_; ++c) {
        for (int g = off_[c]; g < off_[c + 1]; ++g) cid[g] = c;
        poff[c] = ptot;
        const int nj_pad = (n_[c] + tile_of(kmode_) - 1) / tile_of(kmode_) * tile_of(kmode_);
        ptot += (long long)n_[c] * batch_max_split(kmode_, nj_pad, min_tiles_);
    }
    auto alloc = [&](void **p, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(p, bytes > 0 ? bytes : 16);
        if (e == cudaSuccess) {
            allocs_.push_back(*p);
            cudaMemsetAsync(*p, 0, bytes > 0 ? bytes : 16, stream_);
        }
        return e;
    };
    const size_t N = ntot_;
    void *p;
    ECHK(alloc(&p, sizeof(int) * (nc_ + 1)), "alloc"); d_.off = (int *)p;
    ECHK(alloc(&p, sizeof(int) * nc_), "alloc"); d_.n = (int *)p;
    ECHK(alloc(&p, sizeof(int) * N), "alloc"); d_.cid = (int *)p;
    ECHK(alloc(&p, sizeof(double) * nc_), "alloc"); d_.eps2 = (double *)p;
    ECHK(alloc(&p, sizeof(FixedScale) * nc_), "alloc"); d_.fs = (FixedScale *)p;
    ECHK(alloc(&p, sizeof(long long) * nc_), "alloc"); d_.part_off = (long long *)p;
    ECHK(alloc(&p, sizeof(double) * 3 * N), "alloc"); d_.x = (double *)p;
    ECHK(alloc(&p, sizeof(double) * 3 * N), "alloc"); d_.v = (double *)p;
    ECHK(alloc(&p, sizeof(double) * 3 * N), "alloc"); d_.a = (double *)p;
    ECHK(alloc(&p, sizeof(double) * 3 * N), "alloc"); d_.jk = (double *)p;
    ECHK(alloc(&p, sizeof(double) * N), "alloc"); d_.t = (double *)p;
    ECHK(alloc(&p, sizeof(double) * N), "alloc"); d_.dt = (double *)p;
    ECHK(alloc(&p, sizeof(double) * N), "alloc"); d_.m = (double *)p;
    ECHK(alloc(&p, sizeof(int) * N), "alloc"); d_.slot = (int *)p;
    ECHK(alloc(&p, sizeof(double) * nc_), "alloc"); d_.tblock = (double *)p;
    ECHK(alloc(&p, sizeof(int) * nc_), "alloc"); d_.count = (int *)p;
    ECHK(alloc(&p, sizeof(int) * nc_), "alloc"); d_.ntask = (int *)p;
    ECHK(alloc(&p, sizeof(JRecF64) * N), "alloc"); d_.jrec = p;
    ECHK(alloc(&p, sizeof(IRec) * N), "alloc"); d_.irec = (IRec *)p;
    ECHK(alloc(&p, sizeof(double) * 3 * N), "alloc"); d_.acc1 = (double *)p;
    ECHK(alloc(&p, sizeof(double) * 3 * N), "alloc"); d_.jerk1 = (double *)p;
    ECHK(alloc(&p, sizeof(double) * N), "alloc"); d_.pot1 = (double *)p;
    ECHK(alloc(&p, sizeof(int) * N), "alloc"); d_.nn1 = (int *)p;
    ECHK(alloc(&p, sizeof(Partial) * (size_t)ptot), "alloc"); d_.part = (Partial *)p;
    ECHK(alloc(&p, sizeof(ForceParams) * nc_), "alloc"); d_.items = (ForceParams *)p;
    ECHK(alloc(&p, sizeof(int) * (nc_ + 1)), "alloc"); d_.task0 = (int *)p;
    ECHK(alloc(&p, sizeof(int) * (nc_ + 1)), "alloc"); d_.ipre = (int *)p;
    ECHK(alloc(&p, sizeof(int) * 4), "alloc"); d_.counter = (int *)p;
    ECHK(alloc(&p, sizeof(int) * nc_), "alloc"); d_.order = (int *)p;
    ECHK(alloc(&p, sizeof(unsigned long long) * nc_), "alloc"); d_.tnext = (unsigned long long *)p;
    ECHK(alloc(&p, sizeof(unsigned)), "alloc"); d_.done = (unsigned *)p;
    ECHK(alloc(&p, sizeof(int) * N), "alloc"); d_.tcnt = (int *)p;
    ECHK(alloc(&p, sizeof(unsigned) * 4), "alloc"); d_.status = (unsigned *)p;
    ECHK(alloc(&p, sizeof(int) * 4), "alloc"); d_.active = (int *)p;
    ECHK(alloc(&p, sizeof(unsigned long long) * 2), "alloc"); d_.interactions = (unsigned long long *)p;
    d_.nc = nc_;
    d_.ntot = ntot_;
    d_.eta = eta_;
    d_.eta_s = 0.01;
    d_.dt_max = 1.0 / 16;
    d_.kmode = kmode_;
    d_.cfg = batch_config(kmode_);
    // The shape the tuner settles on for this engine's workloads (64 i per
    // CTA, 592 tasks per cluster), also the untuned default: with the
    // servers' work cap instead the bench's ensemble ran 249-270 us per
    // iteration against 225.
    d_.cfg.nsplit = 592;
    d_.cfg.min_tiles = min_tiles_;
    ctas_ = batch_ctas(kmode_, d_.cfg, num_sms_);
    ECHK(cudaMemcpyAsync((void *)d_.off, off_.data(), sizeof(int) * (nc_ + 1), cudaMemcpyHostToDevice, stream_), "copy");
    ECHK(cudaMemcpyAsync((void *)d_.n, n_.data(), sizeof(int) * nc_, cudaMemcpyHostToDevice, stream_), "copy");
    ECHK(cudaMemcpyAsync((void *)d_.cid, cid.data(), sizeof(int) * N, cudaMemcpyHostToDevice, stream_), "copy");
    ECHK(cudaMemcpyAsync((void *)d_.eps2, eps2_.data(), sizeof(double) * nc_, cudaMemcpyHostToDevice, stream_), "copy");
    ECHK(cudaMemcpyAsync((void *)d_.part_off, poff.data(), sizeof(long long) * nc_, cudaMemcpyHostToDevice, stream_),
         "copy");
    hm_.assign(N, 0.0);
    hx_.assign(3 * N, 0.0);
    hv_.assign(3 * N, 0.0);
    ECHK(cudaStreamSynchronize(stream_), "sync");
    return 0;
}

int Ensemble::set_cluster(int c, const double *m, const double (*x)[3], const double (*v)[3]) {
    if (c < 0 || c >= nc_) {
        err = "ensemble: cluster index out of range";
        return -1;
    }
    const int o = off_[c], N = ntot_;
    for (int i = 0; i < n_[c]; ++i) {
        hm_[o + i] = m[i];
        for (int q = 0; q < 3; ++q) {
            hx_[q * N + o + i] = x[i][q];
            hv_[q * N + o + i] = v[i][q];
        }
    }
    return 0;
}

int Ensemble::push_host_state() {
    const size_t N = ntot_;
    ECHK(cudaMemcpyAsync(d_.m, hm_.data(), sizeof(double) * N, cudaMemcpyHostToDevice, stream_), "copy");
    ECHK(cudaMemcpyAsync(d_.x, hx_.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice, stream_), "copy");
    ECHK(cudaMemcpyAsync(d_.v, hv_.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice, stream_), "copy");
    ECHK(cudaMemsetAsync(d_.t, 0, sizeof(double) * N, stream_), "memset");
    ECHK(cudaMemsetAsync(d_.a, 0, sizeof(double) * 3 * N, stream_), "memset");
    ECHK(cudaMemsetAsync(d_.jk, 0, sizeof(double) * 3 * N, stream_), "memset");
    // fixed-point range per cluster: |x| < 2^(E-2), margin 4 for the motion
    std::vector<FixedScale> fs(nc_);
    for (int c = 0; c < nc_; ++c) {
        double xm = 0;
        for (int q = 0; q < 3; ++q)
            for (int i = 0; i < n_[c]; ++i) xm = std::max(xm, std::fabs(hx_[q * N + off_[c] + i]));
        const int E = xm > 0 ? std::ilogb(xm) + 3 : 1;
        fs[c].to_units = std::ldexp(1.0, 23 - E);
        fs[c].hi_unit = std::ldexp(1.0, E - 23);
        fs[c].lo_unit = std::ldexp(1.0, E - 46);
    }
    ECHK(cudaMemcpyAsync((void *)d_.fs, fs.data(), sizeof(FixedScale) * nc_, cudaMemcpyHostToDevice, stream_), "copy");
    ECHK(cudaStreamSynchronize(stream_), "sync");
    return 0;
}

// One iteration: schedule (unless fused), predict, scan, force and
// (mode != 2) the corrector.  fused: block steps after the first of a run,
// whose block times and members come from the previous corrector and the
// predict kernel (mode 0 only).
int Ensemble::iteration(int mode, bool fused) {
    fused = fused && fuse_ && mode == 0;
    if (!fused) ens_schedule_kernel<<<nc_, kSchedThreads, 0, stream_>>>(d_, mode);
    const int per = kmode_ == kKernMixedP ? 2 : 1;
    const int units = (ntot_ / per + 255) / 256;
    ens_predict_kernel<<<units, 256, 0, stream_>>>(d_, fused ? 1 : 0);
    ens_scan_kernel<<<1, 1024, 0, stream_>>>(d_);
    BatchArgs ba;
    ba.items = d_.items;
    ba.task0 = d_.task0;
    ba.ipre = d_.ipre;
    ba.n_items = nc_;
    ba.H = d_.cfg.H;
    ba.counter = d_.counter;
    ba.one_task_per_cta = 0;
    ba.order = d_.order;
    // total_i = 0: the splits are folded inside the force kernel (tile_counter)
    cudaError_t e = launch_force_batch(stream_, kmode_, d_.cfg, ba, ctas_, 0, false, true);
    if (e != cudaSuccess) return fail("force launch", e);
    if (mode != 2) ens_correct_kernel<<<4 * num_sms_, 256, 0, stream_>>>(d_, mode);
    launches_ += (fused ? 3 : 4) + (mode != 2 ? 1 : 0);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int Ensemble::start() {
    if (push_host_state()) return -1;
    if (iteration(1)) return -1;
    ECHK(cudaStreamSynchronize(stream_), "start");
    unsigned long long z = 0;
    ECHK(cudaMemcpy(d_.interactions, &z, sizeof z, cudaMemcpyHostToDevice), "copy");
    return 0;
}

int Ensemble::run_batched(double t_end, EnsembleStats *st, int tune) {
    ECHK(cudaSetDevice(device_), "device");
    d_.t_end = t_end;
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    unsigned long long i0 = 0, l0 = 0;
    ECHK(cudaMemcpy(&i0, d_.interactions, sizeof i0, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(&l0, d_.interactions + 1, sizeof l0, cudaMemcpyDeviceToHost), "copy");
    ens_cap_kernel<<<(ntot_ + 255) / 256, 256, 0, stream_>>>(d_);
    ECHK(cudaStreamSynchronize(stream_), "cap");
    auto t0 = std::chrono::steady_clock::now();
    const long long launches0 = launches_;
    // The run's first block step goes through the schedule kernel (the steps
    // were capped at t_end since the last corrector); the rest are fused.
    if (iteration(0, false)) return -1;
    long long iters = 1;
    // Events and the pinned flag word are released on every return.
    struct Scratch {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        int *h_active = nullptr;
        ~Scratch() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            if (h_active) cudaFreeHost(h_active);
        }
    } sc;
    // Autotune the launch shape on the first iterations of the run: the
    // i-tile of large blocks (H warps per j-tile: i per CTA = 256 / H) and
    // the j-split factor (tasks wanted per cluster), by measured time per
    // iteration on the live integration.
    if (tune) {
        const int hs[4] = {8, 4, 2, 1};
        const int targets[3] = {296, 592, 1184};
        double best = 1e30;
        int bestH = d_.cfg.H, bestT = d_.cfg.nsplit;
        ECHK(cudaEventCreate(&sc.e0), "event");
        ECHK(cudaEventCreate(&sc.e1), "event");
        cudaEvent_t e0 = sc.e0, e1 = sc.e1;
        for (int tt : targets) {
            for (int h : hs) {
                d_.cfg.H = h;
                d_.cfg.nsplit = tt;
                ctas_ = batch_ctas(kmode_, d_.cfg, num_sms_);
                cudaEventRecord(e0, stream_);
                for (int k = 0; k < 8; ++k)
                    if (iteration(0, true)) return -1;
                cudaEventRecord(e1, stream_);
                cudaEventSynchronize(e1);
                iters += 8;
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) {
                    best = ms;
                    bestH = h;
                    bestT = tt;
                }
            }
        }
        d_.cfg.H = bestH;
        d_.cfg.nsplit = bestT;
        ctas_ = batch_ctas(kmode_, d_.cfg, num_sms_);
    }
    if (st) {
        st->tuned_h = d_.cfg.H;
        st->tuned_tasks = d_.cfg.nsplit > 0 ? d_.cfg.nsplit : 592;
    }
    // Capture K iterations as one graph.
    const int K = 8;
    cudaGraph_t g;
    const long long launches_before_capture = launches_;
    ECHK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
    for (int k = 0; k < K; ++k) iteration(0, true);
    ECHK(cudaStreamEndCapture(stream_, &g), "capture");
    const long long launches_per_graph = launches_ - launches_before_capture;
    launches_ = launches_before_capture;
    ECHK(cudaGraphInstantiate(&graph_, g, 0), "instantiate");
    cudaGraphDestroy(g);
    // Two graph launches in flight: while the GPU runs one, the host waits
    // for the other's active-cluster count, so the GPU never idles on the
    // host's check.  Once every cluster has finished, the launch already in
    // flight runs iterations with no active cluster (no work, no change).
    ECHK(cudaMallocHost(&sc.h_active, 2 * sizeof(int)), "pinned");
    int *h_active = sc.h_active;
    cudaEvent_t done[2];
    for (cudaEvent_t &e : done) ECHK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    struct Events {
        cudaEvent_t *e;
        ~Events() {
            cudaEventDestroy(e[0]);
            cudaEventDestroy(e[1]);
        }
    } ev_guard{done};
    auto launch = [&](int slot) -> int {
        ECHK(cudaGraphLaunch(graph_, stream_), "graph launch");
        iters += K;
        launches_ += launches_per_graph;
        ECHK(cudaMemcpyAsync(h_active + slot, d_.active, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy");
        ECHK(cudaEventRecord(done[slot], stream_), "event");
        return 0;
    };
    if (launch(0)) return -1;
    for (int slot = 0;; slot ^= 1) {
        if (launch(slot ^ 1)) return -1;
        ECHK(cudaEventSynchronize(done[slot]), "run");
        if (h_active[slot] == 0) break;
        if (iters > max_iters_ ||
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > max_seconds_) {
            cudaStreamSynchronize(stream_);
            err = "ensemble: iteration or time limit reached";
            return -1;
        }
    }
    ECHK(cudaStreamSynchronize(stream_), "run");
    auto t1 = std::chrono::steady_clock::now();
    unsigned long long i1 = 0, l1 = 0;
    unsigned status = 0;
    ECHK(cudaMemcpy(&i1, d_.interactions, sizeof i1, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(&l1, d_.interactions + 1, sizeof l1, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(&status, d_.status, sizeof status, cudaMemcpyDeviceToHost), "copy");
    if (status) {
        err = "ensemble: device status " + std::to_string(status) + " (fixed-point range or copy timeout)";
        return -2;
    }
    if (st) {
        st->seconds = std::chrono::duration<double>(t1 - t0).count();
        st->interactions = (long long)(i1 - i0);
        st->lane_interactions = (long long)(l1 - l0);
        st->iterations = iters;
        st->launches = launches_ - launches0;
    }
    return 0;
}

int Ensemble::sync_host_state() {
    const size_t N = ntot_;
    sx_.resize(3 * N); sv_.resize(3 * N); sa_.resize(3 * N); sj_.resize(3 * N);
    st_.resize(N); sdt_.resize(N); sm_.resize(N);
    ECHK(cudaMemcpy(sx_.data(), d_.x, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(sv_.data(), d_.v, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(sa_.data(), d_.a, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(sj_.data(), d_.jk, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(st_.data(), d_.t, sizeof(double) * N, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(sdt_.data(), d_.dt, sizeof(double) * N, cudaMemcpyDeviceToHost), "copy");
    ECHK(cudaMemcpy(sm_.data(), d_.m, sizeof(double) * N, cudaMemcpyDeviceToHost), "copy");
    return 0;
}

// The plain engine: one g6 engine instance per cluster, one
// firsthalf/lasthalf call per cluster per block, host-side prediction and
// correction (kira's own pattern), clusters taking turns.
int Ensemble::run_per_cluster(double t_end, EnsembleStats *st) {
    if (sync_host_state()) return -1;
    const int N = ntot_;
    for (int g = 0; g < N; ++g)
        while (sdt_[g] > kDtMin && st_[g] < t_end && st_[g] + sdt_[g] > t_end) sdt_[g] *= 0.5;
    std::vector<Engine *> eng(nc_, nullptr);
    int maxn = 0;
    for (int c = 0; c < nc_; ++c) maxn = std::max(maxn, n_[c]);
    for (int c = 0; c < nc_; ++c) {
        Engine *e = new Engine(100000 + c);
        eng[c] = e;
        if (e->open(device_, n_[c]) || e->set_mode(mode_) || e->set_npipes(maxn)) {
            err = "ensemble baseline: " + e->last_error;
            for (Engine *x : eng) delete x;
            return -1;
        }
        const int o = off_[c];
        for (int i = 0; i < n_[c]; ++i) {
            const int g = o + i;
            double xx[3], vv[3], a2[3], j6[3];
            for (int q = 0; q < 3; ++q) {
                xx[q] = sx_[q * N + g];
                vv[q] = sv_[q * N + g];
                a2[q] = 0.5 * sa_[q * N + g];
                j6[q] = sj_[q * N + g] / 6.0;
            }
            e->set_j(i, i, st_[g], sm_[g], nullptr, j6, a2, vv, xx);
        }
    }
    std::vector<int> idx(maxn);
    std::vector<double> xi(3 * (size_t)maxn), vi(3 * (size_t)maxn), acc(3 * (size_t)maxn), jerk(3 * (size_t)maxn),
        pot(maxn);
    std::vector<int> nn(maxn);
    long long inter = 0, iters = 0, launches0 = 0;
    for (Engine *e : eng) launches0 += e->stats().launches;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<char> done(nc_, 0);
    int active = nc_;
    int rc = 0;
    while (active > 0 && rc == 0) {
        ++iters;
        if (iters > max_iters_ ||
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > max_seconds_) {
            err = "ensemble baseline: iteration or time limit reached";
            rc = -1;
            break;
        }
        for (int c = 0; c < nc_ && rc == 0; ++c) {
            if (done[c]) continue;
            const int o = off_[c], n = n_[c];
            double tb = DBL_MAX;
            for (int i = 0; i < n; ++i) tb = std::min(tb, st_[o + i] + sdt_[o + i]);
            if (tb > t_end) {
                done[c] = 1;
                --active;
                continue;
            }
            int ni = 0;
            for (int i = 0; i < n; ++i) {
                const int g = o + i;
                if (st_[g] + sdt_[g] != tb) continue;
                const double h = tb - st_[g];
                for (int q = 0; q < 3; ++q) {
                    const double a2 = 0.5 * sa_[q * N + g], j6 = sj_[q * N + g] * (1.0 / 6.0);
                    xi[3 * ni + q] = sx_[q * N + g] + h * (sv_[q * N + g] + h * (a2 + h * j6));
                    vi[3 * ni + q] = sv_[q * N + g] + h * (2.0 * a2 + h * (3.0 * j6));
                }
                idx[ni++] = i;
            }
            Engine *e = eng[c];
            e->set_ti(tb);
            if (e->firsthalf(n, ni, idx.data(), (const double(*)[3])xi.data(), (const double(*)[3])vi.data(),
                             eps2_[c], nullptr) ||
                e->lasthalf(ni, (double(*)[3])acc.data(), (double(*)[3])jerk.data(), pot.data(), nn.data())) {
                err = "ensemble baseline: " + e->last_error;
                rc = -1;
                break;
            }
            inter += (long long)ni * n;
            for (int k = 0; k < ni; ++k) {
                const int g = o + idx[k];
                const double h = tb - st_[g], h2 = h * h, h3 = h2 * h;
                double sa1 = 0, sj1 = 0, sa2 = 0, sa3 = 0;
                double xn[3], vn[3], a2h[3], j6h[3];
                for (int q = 0; q < 3; ++q) {
                    const double a0 = sa_[q * N + g], j0 = sj_[q * N + g];
                    const double a1 = acc[3 * k + q], j1 = jerk[3 * k + q];
                    const double sn = (-6.0 * (a0 - a1) - h * (4.0 * j0 + 2.0 * j1)) / h2;
                    const double cr = (12.0 * (a0 - a1) + 6.0 * h * (j0 + j1)) / h3;
                    xn[q] = xi[3 * k + q] + h2 * h2 * (sn / 24.0 + h * cr / 120.0);
                    vn[q] = vi[3 * k + q] + h3 * (sn / 6.0 + h * cr / 24.0);
                    const double a2e = sn + h * cr;
                    sa1 += a1 * a1;
                    sj1 += j1 * j1;
                    sa2 += a2e * a2e;
                    sa3 += cr * cr;
                    sx_[q * N + g] = xn[q];
                    sv_[q * N + g] = vn[q];
                    sa_[q * N + g] = a1;
                    sj_[q * N + g] = j1;
                    a2h[q] = 0.5 * a1;
                    j6h[q] = j1 / 6.0;
                }
                const double den = std::sqrt(sj1) * std::sqrt(sa3) + sa2;
                double dtn = den > 0 ? std::sqrt(eta_ * (std::sqrt(sa1) * std::sqrt(sa2) + sj1) / den) : 2.0 * h;
                dtn = pow2_floor(std::max(dtn, kDtMin));
                dtn = std::min(dtn, std::min(2.0 * h, d_.dt_max));
                while (dtn > kDtMin && (std::fmod(tb, dtn) != 0.0 || (tb < t_end && tb + dtn > t_end))) dtn *= 0.5;
                st_[g] = tb;
                sdt_[g] = std::max(dtn, kDtMin);
                e->set_j(idx[k], idx[k], tb, sm_[g], nullptr, j6h, a2h, vn, xn);
            }
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    long long launches1 = 0;
    for (Engine *e : eng) {
        launches1 += e->stats().launches;
        delete e;
    }
    if (rc) return rc;
    if (st) {
        st->seconds = std::chrono::duration<double>(t1 - t0).count();
        st->interactions = inter;
        st->iterations = iters;
        st->launches = launches1 - launches0;
    }
    // write the state back so energies/get_cluster see the baseline's result
    ECHK(cudaMemcpy(d_.x, sx_.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice), "copy");
    ECHK(cudaMemcpy(d_.v, sv_.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice), "copy");
    ECHK(cudaMemcpy(d_.a, sa_.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice), "copy");
    ECHK(cudaMemcpy(d_.jk, sj_.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice), "copy");
    ECHK(cudaMemcpy(d_.t, st_.data(), sizeof(double) * N, cudaMemcpyHostToDevice), "copy");
    ECHK(cudaMemcpy(d_.dt, sdt_.data(), sizeof(double) * N, cudaMemcpyHostToDevice), "copy");
    return 0;
}

int Ensemble::energies(double *ek_ep) {
    ECHK(cudaSetDevice(device_), "device");
    if (iteration(2)) return -1;  // all particles, no correction: pot1
    double *d_out = nullptr;
    ECHK(cudaMalloc(&d_out, sizeof(double) * 2 * nc_), "alloc");
    ens_energy_kernel<<<nc_, 256, 0, stream_>>>(d_, d_out);
    cudaError_t e = cudaMemcpyAsync(ek_ep, d_out, sizeof(double) * 2 * nc_, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    cudaFree(d_out);
    if (e != cudaSuccess) return fail("energies", e);
    return 0;
}

int Ensemble::get_cluster(int c, double *m, double (*x)[3], double (*v)[3], double (*acc)[3], double (*jerk)[3],
                          double *t, double *dt) {
    if (c < 0 || c >= nc_) {
        err = "ensemble: cluster index out of range";
        return -1;
    }
    if (sync_host_state()) return -1;
    const int o = off_[c], N = ntot_;
    for (int i = 0; i < n_[c]; ++i) {
        if (m) m[i] = sm_[o + i];
        for (int q = 0; q < 3; ++q) {
            if (x) x[i][q] = sx_[q * N + o + i];
            if (v) v[i][q] = sv_[q * N + o + i];
            if (acc) acc[i][q] = sa_[q * N + o + i];
            if (jerk) jerk[i][q] = sj_[q * N + o + i];
        }
        if (t) t[i] = st_[o + i];
        if (dt) dt[i] = sdt_[o + i];
    }
    return 0;
}

}  // namespace g6

// ---------------------------------------------------------------------------
// C ABI
#include <mutex>
namespace g6 {
void record_error(const std::string &msg);
}
#pragma GCC visibility push(default)
#include "../../include/g6b200.h"
#pragma GCC visibility pop

struct g6b200_ensemble {
    g6::Ensemble *e;
};

extern "C" {

__attribute__((visibility("default"))) g6b200_ensemble *g6b200_ens_create(int nclusters, const int *n,
                                                                         const double *eps2, double eta,
                                                                         int precision, int device) {
    if (nclusters <= 0 || !n || !eps2) return nullptr;
    for (int c = 0; c < nclusters; ++c)
        if (n[c] <= 0) return nullptr;
    auto *e = new g6::Ensemble(nclusters, n, eps2, eta, precision, device);
    if (e->setup()) {
        g6::record_error(e->err);
        delete e;
        return nullptr;
    }
    return new g6b200_ensemble{e};
}

__attribute__((visibility("default"))) int g6b200_ens_set_cluster(g6b200_ensemble *h, int c, const double *m,
                                                                  const double (*x)[3], const double (*v)[3]) {
    int rc = h->e->set_cluster(c, m, x, v);
    if (rc) g6::record_error(h->e->err);
    return rc;
}

__attribute__((visibility("default"))) int g6b200_ens_start(g6b200_ensemble *h) {
    int rc = h->e->start();
    if (rc) g6::record_error(h->e->err);
    return rc;
}

__attribute__((visibility("default"))) int g6b200_ens_run(g6b200_ensemble *h, double t_end, int per_cluster,
                                                          int tune, g6b200_ens_stats *out) {
    g6::EnsembleStats st;
    int rc = per_cluster ? h->e->run_per_cluster(t_end, &st) : h->e->run_batched(t_end, &st, tune);
    if (rc) {
        g6::record_error(h->e->err);
        return rc;
    }
    if (out) {
        out->seconds = st.seconds;
        out->interactions = st.interactions;
        out->iterations = st.iterations;
        out->launches = st.launches;
        out->tuned_h = (int)st.tuned_h;
        out->tuned_tasks = st.tuned_tasks;
        out->lane_interactions = st.lane_interactions;
    }
    return 0;
}

__attribute__((visibility("default"))) int g6b200_ens_energies(g6b200_ensemble *h, double *ek_ep) {
    int rc = h->e->energies(ek_ep);
    if (rc) g6::record_error(h->e->err);
    return rc;
}

__attribute__((visibility("default"))) int g6b200_ens_get_cluster(g6b200_ensemble *h, int c, double *m,
                                                                  double (*x)[3], double (*v)[3], double (*acc)[3],
                                                                  double (*jerk)[3], double *t, double *dt) {
    int rc = h->e->get_cluster(c, m, x, v, acc, jerk, t, dt);
    if (rc) g6::record_error(h->e->err);
    return rc;
}

__attribute__((visibility("default"))) void g6b200_ens_destroy(g6b200_ensemble *h) {
    if (!h) return;
    delete h->e;
    delete h;
}

}  // extern "C"
