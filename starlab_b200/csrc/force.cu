// force.cu -- the i-block x j-particle direct-summation kernel.
//
// Pair terms are those of the reference's accumulate_acc_and_jerk
// (src/node/dyn/hdyn/evolve/hdyn_ev.C:2019-2036): with dr = x_j - x_i,
// dv = v_j - v_i, r2 = dr.dr + eps2,
//     pot -= m/r,  acc += m dr / r^3,  jerk += m/r^3 (dv - 3 (dr.dv)/r2 dr),
// self excluded by index; the nearest neighbour is the first address with
// the smallest dr.dr (no softening; hdyn_inline.C:34-77).
//
// GRAPE-4 variant (FP64 only, kVarG4): the pipeline of the reference's
// GRAPE-4 simulator (src/harpsims/harp3fastsim.c:240-300): per-i softening,
// r2 = dr.dr + eps2_i; a pair contributes only when r2 > 0 (no exclusion by
// index: kira stores the block's own particles at the block time, so self
// has dr = 0 exactly); neighbour test r2 < h2_i on the softened r2.
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
// fixed-point positions, Newton-refined rsqrt.approx); each thread sums up
// to kFlush pair terms in FP32 and then folds them into FP64 totals.  The
// paired layout evaluates two j per FP32x2 instruction (add/mul/fma.f32x2),
// halving the issue slots per interaction.  FP64 mode does the pair
// arithmetic and the sums in FP64.
#include <algorithm>
#include <cfloat>
#include "common.cuh"
#include "force_device.cuh"
#include "kernels.h"

namespace g6 {


int tile_size(int kmode) { return kmode == kKernF64 ? Traits<kKernF64>::T : 256; }

static int units_per_tile(int kmode) { return kmode == kKernMixedP ? Traits<kKernMixedP>::U : tile_size(kmode); }

size_t jrec_bytes(int kmode) {
    switch (kmode) {
        case kKernF64: return sizeof(JRecF64);
        case kKernMixedP: return sizeof(JPairMixed) / 2;
        default: return sizeof(JRecMixed);
    }
}

// ----------------------------------------------------------------------------

// One call: gridDim.x i-tiles x gridDim.y j-splits, one task per CTA.
template <int K, int IL, int R, bool NB, bool IDENT, int V>
__global__ void __launch_bounds__(256, MinBlocks<K, R>::value) force_kernel(const ForceParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    init_bars(smem);
    int gt = 0;
    process_task<K, IL, R, NB, IDENT, V>(p, blockIdx.x, blockIdx.y, smem, gt);
}

// Many calls in one launch: items[k] is one call (its own j-memory,
// i-records, softening, fixed-point scale and outputs); its tasks are
// n_itiles(k) x nsplit(k), numbered from task0[k].  Persistent form: CTAs
// take tasks from a global counter until the list is exhausted.  With
// one_task_per_cta, CTA b runs task b (so CTAs of other launches can be
// scheduled as these retire).
template <int K, int IL, int R, bool NB, bool IDENT, int V>
__global__ void __launch_bounds__(256, MinBlocks<K, R>::value) batch_force_kernel(const BatchArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_task;
    init_bars(smem);
    const int itile = (blockDim.x >> 5) / a.H * IL * R;
    const int total = a.task0[a.n_items];
    int gt = 0;
    for (int it = 0;; ++it) {
        __syncthreads();
        if (threadIdx.x == 0) s_task = a.one_task_per_cta ? (it == 0 ? (int)blockIdx.x : total) : atomicAdd(a.counter, 1);
        __syncthreads();
        const int task = s_task;
        if (task >= total) break;
        int lo = 0, hi = a.n_items - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.task0[mid] <= task) lo = mid; else hi = mid - 1;
        }
        const ForceParams p = a.items[a.order ? a.order[lo] : lo];
        const int local = task - a.task0[lo];
        const int il = batch_il(p.ni);  // the item's lane shape (its H is in p.H)
        bool ok;
        if (il == 32) {
            const int n_itiles = (p.ni + itile - 1) / itile;
            ok = process_task<K, IL, R, NB, IDENT, V>(p, local % n_itiles, local / n_itiles, smem, gt);
        } else if (il == 8) {
            const int it8 = (blockDim.x >> 5) / p.H * 8;
            const int n_itiles = (p.ni + it8 - 1) / it8;
            ok = process_task<K, 8, 1, NB, IDENT, V>(p, local % n_itiles, local / n_itiles, smem, gt);
        } else {
            const int it1 = (blockDim.x >> 5) / p.H;
            const int n_itiles = (p.ni + it1 - 1) / it1;
            ok = process_task<K, 1, 1, NB, IDENT, V>(p, local % n_itiles, local / n_itiles, smem, gt);
        }
        // After a timed-out copy wait this CTA's barrier phases no longer
        // match its tile count: it takes no further task (the status word
        // already reports the failure; the other CTAs finish the list).
        if (!ok) break;
    }
}

// Split reduction for every i of every item with nsplit > 1; ipre[k] is the
// prefix sum of the items' ni (read on the device, so a launch captured in a
// graph serves batches of any size: grid-stride over ipre[n_items]).
__global__ void batch_reduce_kernel(const BatchArgs a) {
    const int total = a.ipre[a.n_items];
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < total; gi += gridDim.x * blockDim.x) {
        int lo = 0, hi = a.n_items - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.ipre[mid] <= gi) lo = mid; else hi = mid - 1;
        }
        const ForceParams &p = a.items[lo];
        if (p.nsplit <= 1) continue;
        const int i = gi - a.ipre[lo];
        Partial q = p.part[i];
        for (int s = 1; s < p.nsplit; ++s) add_partial(q, p.part[(size_t)s * p.ni + i]);
        write_final(p, i, q);
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

template <int K, int IL, int R>
static KernelFn pick3(bool nb, bool ident) {
    // the single-call paired mixed kernels also accumulate the refinement's
    // error indicators
    constexpr int V = kVarUnroll4 | (K == kKernMixedP ? kVarStats : 0);
    if (nb) return ident ? force_kernel<K, IL, R, true, true, V> : force_kernel<K, IL, R, true, false, V>;
    return ident ? force_kernel<K, IL, R, false, true, V> : force_kernel<K, IL, R, false, false, V>;
}

template <int K>
static KernelFn pick2(int il, int r, bool nb, bool ident) {
    if (il == 32) {
        if (K == kKernMixedDS && r == 4) return pick3<K, 32, 4>(nb, ident);
        if (K != kKernMixedP && r == 2) return pick3<K, 32, 2>(nb, ident);
        return pick3<K, 32, 1>(nb, ident);
    }
    if (il == 8) return pick3<K, 8, 1>(nb, ident);
    return pick3<K, 1, 1>(nb, ident);
}

// GRAPE-4 pipeline: FP64 layout, no index identity.
static KernelFn pick_g4(int il, int r, bool nb) {
    constexpr int K = kKernF64, V = kVarG4;
    if (il == 32 && r == 2) return nb ? force_kernel<K, 32, 2, true, false, V> : force_kernel<K, 32, 2, false, false, V>;
    if (il == 32) return nb ? force_kernel<K, 32, 1, true, false, V> : force_kernel<K, 32, 1, false, false, V>;
    if (il == 8) return nb ? force_kernel<K, 8, 1, true, false, V> : force_kernel<K, 8, 1, false, false, V>;
    return nb ? force_kernel<K, 1, 1, true, false, V> : force_kernel<K, 1, 1, false, false, V>;
}

// Potential only (energy sweeps): one i per thread, no neighbour lists.
template <int K>
static KernelFn pick_pot(int il, bool ident) {
    constexpr int V = kVarUnroll4 | kVarPot;
    if (il == 32) return ident ? force_kernel<K, 32, 1, false, true, V> : force_kernel<K, 32, 1, false, false, V>;
    if (il == 8) return ident ? force_kernel<K, 8, 1, false, true, V> : force_kernel<K, 8, 1, false, false, V>;
    return ident ? force_kernel<K, 1, 1, false, true, V> : force_kernel<K, 1, 1, false, false, V>;
}

static KernelFn pick(int kmode, int il, int r, bool nb, bool ident) {
    if (kmode == kKernMixedP) return pick2<kKernMixedP>(il, r, nb, ident);
    if (kmode == kKernMixedDS) return pick2<kKernMixedDS>(il, r, nb, ident);
    return pick2<kKernF64>(il, r, nb, ident);
}

static size_t smem_bytes(int kmode, const ForceConfig &c) {
    size_t tiles = 2 * (size_t)tile_size(kmode) * jrec_bytes(kmode);  // bytes per j x j per tile
    size_t itile = (size_t)(c.warps / c.H) * c.il * c.r;
    size_t red = c.H > 1 ? (size_t)c.H * itile * sizeof(Partial) : 0;
    return 128 + (tiles > red ? tiles : red);
}

size_t partial_bytes(const ForceConfig &cfg, int ni) {
    return cfg.nsplit > 1 ? (size_t)cfg.nsplit * ni * sizeof(Partial) : 0;
}

size_t partial_bytes_fixed(int jper, int nj_pad, int ni) {
    const int nsplit = std::max(1, (nj_pad + jper - 1) / jper);
    return (size_t)nsplit * ni * sizeof(Partial);
}

ForceConfig choose_config(int kmode, int ni, int nj_pad, int num_sms, bool nb) {
    (void)nb;
    ForceConfig c;
    c.warps = kMaxWarps;
    c.il = ni >= 32 ? 32 : (ni > 1 ? 8 : 1);
    if (c.il == 8 && ni > 8) c.il = 32;
    // Register blocking: the scalar mixed layout gains from 2 i per thread,
    // and so does FP64 (two independent FP64 chains per thread hide part of
    // the dependency waits: 10.48 vs 10.58 ms for 16384 x 262144); the
    // paired layout already reuses each loaded j-pair twice and runs out of
    // registers at 2 (measured: 91 ms vs 95 ms for the N = 262144 sweep).
    c.r = ((kmode == kKernMixedDS || kmode == kKernF64) && c.il == 32 && ni >= 8192) ? 2 : 1;
    // i-groups per CTA: at most an eighth of the i-block per CTA, so that a
    // mid-size block spreads over several i-tiles instead of one i-tile
    // split many ways -- whose split fold (one thread per i over all splits)
    // then dominates.  Measured at nj = 262144 (mixed): ni = 256 0.12 vs
    // 0.31 ms, ni = 1024 0.39 vs 0.43 ms; ni >= 2048 unchanged (8 groups).
    int groups_needed = (ni + c.il * c.r - 1) / (c.il * c.r);
    int G = 1;
    while (G * 2 <= c.warps && G * 2 * 8 <= groups_needed) G *= 2;
    c.H = c.warps / G;
    const int T = tile_size(kmode);
    const int JL = 32 / c.il;
    const int U = units_per_tile(kmode);
    while (c.H > 1 && U / (c.H * JL) < 1) c.H /= 2;  // keep >= 1 record per thread per tile
    G = c.warps / c.H;
    const int itile = G * c.il * c.r;
    const int n_itiles = (ni + itile - 1) / itile;
    const int ntiles = nj_pad / T;
    // Fill the GPU with whole waves: 2 resident CTAs per SM, or one per SM
    // for blocks of up to 128 i (fewer splits to fold: ni = 64 0.051 vs
    // 0.062 ms, ni = 16 0.042 vs 0.058 ms).
    const int slots = (ni <= 128 ? 1 : 2) * num_sms;
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

// ---- batched (multi-item persistent) launches

using BatchFn = void (*)(const BatchArgs);

template <int K>
static BatchFn pick_batch(bool nb, bool ident) {
    constexpr int V = kVarUnroll4;
    if (nb) return ident ? batch_force_kernel<K, 32, 1, true, true, V> : batch_force_kernel<K, 32, 1, true, false, V>;
    return ident ? batch_force_kernel<K, 32, 1, false, true, V> : batch_force_kernel<K, 32, 1, false, false, V>;
}

static BatchFn pick_batch(int kmode, bool nb, bool ident) {
    if (kmode == kKernMixedP) return pick_batch<kKernMixedP>(nb, ident);
    if (kmode == kKernMixedDS) return pick_batch<kKernMixedDS>(nb, ident);
    return pick_batch<kKernF64>(nb, ident);
}

ForceConfig batch_config(int kmode) {
    (void)kmode;
    ForceConfig c;
    c.il = 32;
    c.r = 1;
    c.warps = kMaxWarps;
    c.H = 4;
    c.nsplit = 0;
    return c;
}

int batch_ctas(int kmode, const ForceConfig &cfg, int num_sms) {
    int per_sm = 0;
    BatchFn fn = pick_batch(kmode, false, true);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * cfg.warps, smem_bytes(kmode, cfg));
    if (per_sm < 1) per_sm = 1;
    return per_sm * num_sms;
}

cudaError_t launch_force_batch(cudaStream_t s, int kmode, const ForceConfig &cfg, const BatchArgs &a, int ctas,
                               int total_i, bool nb, bool ident) {
    if (a.n_items <= 0) return cudaSuccess;
    BatchFn fn = pick_batch(kmode, nb, ident);
    fn<<<ctas, 32 * cfg.warps, smem_bytes(kmode, cfg), s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (total_i > 0) {
        batch_reduce_kernel<<<std::min((total_i + 255) / 256, 1184), 256, 0, s>>>(a);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_force(cudaStream_t s, int kmode, const ForceConfig &cfg, ForceParams p,
                         bool ident, bool nb, bool g4, bool pot) {
    if (g4 && (kmode != kKernF64 || !p.ieps2)) return cudaErrorInvalidValue;
    if (pot && (g4 || nb || cfg.r != 1 || kmode == kKernMixedDS)) return cudaErrorInvalidValue;
    const int T = tile_size(kmode);
    const int ntiles = p.nj_pad / T;
    if (p.ni <= 0) return cudaSuccess;
    if (cfg.jper > 0) {
        if (cfg.jper % T) return cudaErrorInvalidValue;
        p.jper = cfg.jper;
        p.nsplit = std::max(1, (p.nj_pad + cfg.jper - 1) / cfg.jper);
    } else if (ntiles <= 0) {
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
    KernelFn fn = pot ? (kmode == kKernF64 ? pick_pot<kKernF64>(cfg.il, ident) : pick_pot<kKernMixedP>(cfg.il, ident))
                      : g4 ? pick_g4(cfg.il, cfg.r, nb) : pick(kmode, cfg.il, cfg.r, nb, ident);
    size_t sm = smem_bytes(kmode, cfg);
    fn<<<grid, block, sm, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (p.nsplit > 1 && !p.tile_counter && !p.keep_partials) {
        reduce_partials_kernel<<<(p.ni + 255) / 256, 256, 0, s>>>(p);
        e = cudaGetLastError();
    }
    return e;
}

// Self-test of the bounded wait that guards every j-tile copy: one thread
// waits on an mbarrier that nothing arrives at and no copy completes, so
// the wait runs out after limit_ns and the status word gets the same bit a
// force call sets when a copy wait times out.  No copy is in flight when it
// gives up.
__global__ void copy_wait_selftest_kernel(unsigned *status, unsigned long long limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_barrier_init();
    if (!mbar_wait_bounded(&bar, 0, limit_ns)) atomicOr(status, ST_TMA_TIMEOUT);
}

void launch_copy_wait_selftest(cudaStream_t s, unsigned *status, unsigned long long limit_ns) {
    copy_wait_selftest_kernel<<<1, 32, 0, s>>>(status, limit_ns);
}

}  // namespace g6
