// kernels.h -- launch interfaces between the engine (host) and the kernels.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace g6 {

// Precision modes (public, g6b200_set_precision).
constexpr int kModeF64 = 0;
constexpr int kModeMixed = 1;
// Kernel layouts: the mixed mode has two record layouts with bit-identical
// pair arithmetic: one j per record (scalar FP32), or pairs of j side by
// side evaluated with FP32x2 instructions (the default).
constexpr int kKernF64 = 0;
constexpr int kKernMixedDS = 1;
constexpr int kKernMixedP = 3;

// Fixed-point scaling of the mixed mode for position exponent E
// (all |x| < 2^E): units of the coarse grid and of the fine grid.
struct FixedScale {
    double to_units;  // 2^(23-E): x * to_units = position in coarse units
    double hi_unit;   // 2^(E-23)
    double lo_unit;   // 2^(E-46)
};

// Split an FP64 position into the coarse/fine FP32 pair (see JRecMixed).
// Returns false when |x| >= 2^E (the pair is then still close to x but the
// difference of two pairs is no longer exact).
__device__ __forceinline__ bool to_fixed_split(double x, const FixedScale &fs, float &hi, float &lo) {
    double xq = x * fs.to_units;
    double fh = floor(xq);
    double rem = xq - fh;  // exact, in [0, 1)
    hi = (float)(fh * fs.hi_unit);
    lo = (float)(floor(rem * 8388608.0) * fs.lo_unit);
    return fabs(fh) <= 8388608.0;
}

struct ForceParams {
    const void *jrec;     // JRecMixed[nj_pad] or JRecF64[nj_pad]
    int nj;               // real j count (addresses [0, nj))
    int nj_pad;           // multiple of the tile size
    int jper;             // j per split (multiple of the tile size)
    int nsplit;           // gridDim.y
    const IRec *irec;     // [ni]
    int ni;
    int H;                // j-subranges per CTA (warps sharing the same i)
    double eps2;
    FixedScale fs;
    Partial *part;        // [nsplit][ni] when nsplit > 1
    double *out_acc;      // [ni][3]   (written directly when nsplit == 1)
    double *out_jerk;     // [ni][3]
    double *out_pot;      // [ni]
    int *out_nn;          // [ni]
    int *nb_count;        // [ni]       (neighbour-list variant)
    int *nb_list;         // [ni][nb_cap]
    int nb_cap;
    int include_self;
    unsigned *status;
    // Per-i-tile arrival counters (zero between calls).  When set and
    // nsplit > 1, the last CTA of an i-tile adds the split partials in split
    // order and writes the results, so no separate reduction launch is needed;
    // it leaves its counter at zero again.
    int *tile_counter;
    // GRAPE-4 calls only (null otherwise): per-i softening eps2_i.  With it
    // the kernel follows the GRAPE-4 pipeline: r2 = dr.dr + eps2_i, pairs
    // with r2 == 0 contribute nothing (no exclusion by index), and the
    // neighbour test is r2 < h2_i on the softened r2.
    const double *ieps2;
    // 1: every split's partial sums stay in part[split][i] (also for one
    // split) and are not folded: the multi-GPU j-split combines them.
    int keep_partials;
    // Mixed-mode error indicators (qa, qj of Partial) per i, [ni][2], when
    // the kernel accumulates them (single-call paired mixed kernels).
    float *out_q;
    // When set: the results of i go to row out_map[i] of the outputs (the
    // refinement's FP64 pass writes its particles' rows of the call's
    // outputs directly).
    const int *out_map;
};

// A batch of calls for the persistent multi-item kernel (device pointers).
struct BatchArgs {
    const ForceParams *items;  // [n_items], each with jper/nsplit/H filled in
    const int *task0;          // [n_items + 1] prefix of n_itiles * nsplit
    const int *ipre;           // [n_items + 1] prefix of ni
    int n_items;
    int H;                     // j-subranges per CTA (same for every item)
    int *counter;              // task counter, zero before the launch
    int one_task_per_cta;      // 1: grid = tasks, CTA b runs task b (no counter)
    // Optional [n_items]: task0 is a prefix over items[order[0]],
    // items[order[1]], ... (the order tasks are handed out in); null = 0, 1, ...
    const int *order = nullptr;
};

struct ForceConfig {
    int il;       // i-lanes per warp (1, 8, 32)
    int r;        // i per thread (1, 2, 4; 2 and 4 only with il = 32)
    int warps;    // warps per CTA
    int H;        // j-subranges per CTA
    int nsplit;   // CTAs along j
    int jper = 0; // > 0: j per split fixed (a multiple of the tile); nsplit follows
    int min_tiles = 4;  // batched plans: fewest j-tiles per split (1, 2, 4 or 8)
};

void launch_scatter(cudaStream_t s, int n, const int *addr, const int *index, const double *vals,
                    double *jraw, int *jindex, int cap);
// Device copies of a caller's j arrays for a bulk upload (addr/index/k18 may
// be null: addresses 0..n-1, index = address, k18 = 0).
struct BulkJ {
    const double *t, *m, *x, *v, *a2, *j6, *k18;
    const int *addr, *index;
};
void launch_scatter_bulk(cudaStream_t s, int n, const BulkJ &b, double *jraw, int *jindex, int cap);
// A small force call's host data, passed by value as the parameter of one
// kernel (so a call of up to kSmallMax i-particles and j-updates needs no
// host->device copy): the staged j-updates (ascending address), the
// i-records, and the prediction to make.
constexpr int kSmallMax = 64;
struct SmallCall {
    int n_upd, ni, nj, nj_pad, cap, predict, parity, g4;
    double ti;
    FixedScale fs;
    int addr[kSmallMax];
    int index[kSmallMax];
    double vals[kSmallMax][JF_COUNT];  // JF_* fields, as the staging records
    IRec irec[kSmallMax];
    double ieps2[kSmallMax];           // GRAPE-4 calls
};
// One launch: apply the updates to the raw j-state, predict j (if
// sc.predict) into jrec, write the i-records (and GRAPE-4 softening), and
// clear status word parity ^ 1 for the next call; range reports go to word
// parity.
void launch_small_call(cudaStream_t s, int kmode, const SmallCall &sc, double *jraw, int *jindex, void *jrec,
                       IRec *irec, double *ieps2, unsigned *status2);
void launch_predict(cudaStream_t s, int kmode, const double *jraw, const int *jindex, int cap,
                    int nj, int nj_pad, double ti, const FixedScale &fs, void *jrec,
                    unsigned *status);

void launch_irec_from_j(cudaStream_t s, const double *jraw, const int *jindex, int cap, int i0, int ni,
                        double ti, IRec *out);

// Energies of a sweep over the stored particles [i0, i0 + ni): epot =
// 1/2 sum m_i pot_i and ekin = 1/2 sum m_i |v_i|^2 with v the i-records'
// (predicted) velocities, masses from the raw j-state; FP64 in a fixed
// order (kEnergyBlocks block partials, then one block).  work holds
// 2 * kEnergyBlocks + 2 doubles; the totals land in work[2 kEnergyBlocks],
// work[2 kEnergyBlocks + 1].
constexpr int kEnergyBlocks = 296;
void launch_energy(cudaStream_t s, int ni, int i0, const IRec *irec, const double *jraw, int cap,
                   const double *pot, double *work);

// kmode: kKernF64 / kKernMixedDS / kKernMixedP.
int tile_size(int kmode);
size_t jrec_bytes(int kmode);
// Choose a launch configuration for ni x nj (heuristic; autotuner overrides).
ForceConfig choose_config(int kmode, int ni, int nj_pad, int num_sms, bool nb);
// Launch force (+ split reduction).  Returns a cudaError_t.  pot: the
// potential only (acc, jerk written as zero, nn as 0); paired mixed or FP64
// layout, cfg.r == 1, no neighbour lists.
cudaError_t launch_force(cudaStream_t s, int kmode, const ForceConfig &cfg, ForceParams p,
                         bool ident, bool nb, bool g4 = false, bool pot = false);
size_t partial_bytes(const ForceConfig &cfg, int ni);
// Partial-sum bytes of a launch whose splits hold jper j each (keep_partials).
size_t partial_bytes_fixed(int jper, int nj_pad, int ni);

// Batched launches.  batch_plan fills jper/nsplit/H of one item from its own
// (ni, nj) only -- never from the rest of the batch -- so an item's sums are
// bit-identical alone and in any mix.  batch_itile is the i-tile of the
// batched kernel.
__host__ __device__ inline int batch_itile(const ForceConfig &cfg) { return cfg.warps / cfg.H * cfg.il * cfg.r; }

__host__ __device__ inline int tile_of(int kmode) { return kmode == kKernF64 ? 128 : 256; }

// Lane shape of one item of a batched launch, from its own ni: blocks of
// 1-2 i run one i per warp group with 32 j-lanes (IL = 1), blocks of up to
// 16 run 8 i-lanes x 4 j-lanes (IL = 8) with every warp on the j-range, and
// larger ones the launch's IL = 32 shape -- so a small block does not leave
// most of a 32-lane i-tile idle.
__host__ __device__ inline int batch_il(int ni) { return ni <= 2 ? 1 : (ni <= 16 ? 8 : 32); }
__host__ __device__ inline int batch_item_H(int kmode, const ForceConfig &cfg, int ni) {
    const int il = batch_il(ni);
    if (il == 32) return cfg.H;
    const int units = kmode == kKernMixedP ? tile_of(kmode) / 2 : tile_of(kmode);  // records per tile
    int h = cfg.warps;
    while (h > 1 && units / (h * (32 / il)) < 1) h /= 2;  // at least one record per lane per tile
    return h;
}
__host__ __device__ inline int batch_item_itile(int kmode, const ForceConfig &cfg, int ni) {
    const int il = batch_il(ni);
    return il == 32 ? batch_itile(cfg) : cfg.warps / batch_item_H(kmode, cfg, ni) * il;
}

// Split rule of the batched kernel: a number of tasks wanted per item that
// depends on the item alone (never on the batch): cfg.nsplit when set, e.g.
// by the ensemble's tuner; else 592 = 4 x 148 but no more than one task per
// kMinTaskWork interactions (the servers: small calls stay in few tasks, so
// a batch of many calls is not cut into tasks too small to keep the
// pipeline busy); at least cfg.min_tiles tiles per split (4 unless the
// ensemble asks for shorter tasks).
constexpr long long kMinTaskWork = 65536;
__host__ __device__ inline void batch_plan(int kmode, const ForceConfig &cfg, ForceParams &item, int &n_tasks) {
    const long long work_cap = ((long long)item.ni * item.nj_pad) / kMinTaskWork;
    const int kTargetTasks = cfg.nsplit > 0 ? cfg.nsplit
                                            : (int)(work_cap < 1 ? 1 : (work_cap < 592 ? work_cap : 592));
    const int T = tile_of(kmode);
    const int ntiles = item.nj_pad / T;
    const int itile = batch_item_itile(kmode, cfg, item.ni);
    const int n_itiles = (item.ni + itile - 1) / itile;
    item.H = batch_item_H(kmode, cfg, item.ni);
    if (item.ni <= 0) {
        item.nsplit = 1;
        item.jper = T;
        n_tasks = 0;
        return;
    }
    if (ntiles <= 0) {
        item.nsplit = 1;
        item.jper = T;
    } else {
        int sp = (kTargetTasks + n_itiles - 1) / n_itiles;
        const int mt = cfg.min_tiles > 1 ? cfg.min_tiles : 1;
        const int cap = (ntiles + mt - 1) / mt;
        sp = sp < cap ? sp : cap;
        sp = sp > 1 ? sp : 1;
        const int per_split_tiles = (ntiles + sp - 1) / sp;
        item.jper = per_split_tiles * T;
        item.nsplit = (ntiles + per_split_tiles - 1) / per_split_tiles;
    }
    n_tasks = n_itiles * item.nsplit;
}

// Largest nsplit batch_plan can choose for nj_pad with at least min_tiles
// tiles per split (sizes the partials).
__host__ __device__ inline int batch_max_split(int kmode, int nj_pad, int min_tiles = 4) {
    const int ntiles = nj_pad / tile_of(kmode);
    const int mt = min_tiles > 1 ? min_tiles : 1;
    const int cap = (ntiles + mt - 1) / mt;
    return cap > 1 ? cap : 1;
}
ForceConfig batch_config(int kmode);
// One persistent launch over all tasks (grid = ctas) + the split reduction
// over total_i i-particles.
// ctas: persistent grid size, or (one_task_per_cta) the total task count.
cudaError_t launch_force_batch(cudaStream_t s, int kmode, const ForceConfig &cfg, const BatchArgs &a, int ctas,
                               int total_i, bool nb, bool ident);
int batch_ctas(int kmode, const ForceConfig &cfg, int num_sms);

// Self-test of the bounded copy wait: a wait on a barrier nothing arrives
// at, which sets ST_TMA_TIMEOUT in *status after limit_ns.
void launch_copy_wait_selftest(cudaStream_t s, unsigned *status, unsigned long long limit_ns);

// Multi-GPU j-split (split.cu): order-independent fixed-point combination
// of per-block partial sums across ranks.  agree [8 ni], sums [7 ni] and
// negj [ni] are int64 device buffers the caller's collectives reduce.
int split_log2_blocks(long long nblocks);
void launch_split_agree(cudaStream_t s, int ni, int nsplit, const Partial *part, long long *agree);
void launch_split_fix(cudaStream_t s, int ni, int nsplit, int g, long long j_offset, const Partial *part,
                      const long long *agree, long long *sums, long long *negj);
void launch_split_finish(cudaStream_t s, int ni, int g, long long nj_total, const long long *agree,
                         const long long *sums, const long long *negj, double *acc, double *jerk, double *pot,
                         int *nn);

// Mixed-mode FP64 refinement (refine.cu): particles whose error indicators
// (ForceParams::out_q) exceed the bounds below are recomputed in FP64.
constexpr double kRefineA = 1.0;  // max (m/r^2) / |acc|
constexpr double kRefineJ = 1.6;  // max (m/r^3) v_rms / |jerk|
constexpr int kRefineBlocks = 256;
struct RefineArgs {
    int ni, nj, nj_pad, ident;
    double eps2;
    const double *v2;         // [kRefineBlocks + 1]: mean |v|^2 of the j-set in the last entry
    const float *q;           // [ni][2] error indicators
    const IRec *irec;         // [ni] the call's i-records
    const void *jrec64;       // JRecF64 [nj_pad] at the call's block time
    double *acc, *jerk, *pot; // the call's outputs, refined in place
    int *nn;
    int *count, *list;        // flagged count (zero between calls), [ni] flagged i
    IRec *irec_ref;           // [ni]
    Partial *part;            // refine_partial_records(ni)
    int *tcnt;                // [ni] i-tile counters, zero between calls
    ForceParams *items;       // [1]
    int *pre;                 // [4]: task and i prefix sums of the FP64 item; pre[3] = flagged count
    int *counter;
    unsigned *done;           // flag blocks finished, zero between calls
    unsigned *status;
};
void launch_refine_v2(cudaStream_t s, const double *jraw, int cap, int nj, double *work);
cudaError_t launch_refine(cudaStream_t s, const RefineArgs &r, int num_sms);
// Tasks wanted by the refinement's FP64 pass over `count` flagged i against
// nj_pad j: one per kMinTaskWork interactions (as the servers' plan), but no
// fewer than kRefineMinTasks -- a call with a handful of flagged particles
// otherwise ran as a dozen CTAs walking long j-ranges (ni = 128: 0.32 ms
// with the refinement vs 0.12 ms without) -- and no more than 592.
constexpr int kRefineMinTasks = 128;
__host__ __device__ inline int refine_tasks_wanted(int count, int nj_pad) {
    const long long wc = (long long)count * nj_pad / kMinTaskWork;
    return (int)(wc < kRefineMinTasks ? kRefineMinTasks : (wc > 592 ? 592 : wc));
}
// Split partial records the FP64 pass of a call of ni i can use: at most
// 592 tasks over i-tiles of at most 64 i, so nsplit x flagged stays below
// 592 x 64 + flagged.
__host__ __device__ inline size_t refine_partial_records(int ni) { return 64 * 600 + (size_t)ni; }

// Neighbour lists: per-i sort + compaction into ascending address order.
// offsets[ni+1] (exclusive scan of min(count, cap)), out[total].
cudaError_t launch_nb_compact(cudaStream_t s, int ni, const int *count, const int *list, int cap,
                              long long *offsets, int *out);
// Full ascending neighbour list of one GRAPE-4 i-record over the predicted
// FP64 j-records (JRecF64[nj]); at most cap entries, *count = hits.
cudaError_t launch_nb_full_g4(cudaStream_t s, const void *jrec, int nj, const IRec &q, double eps2, int *out,
                              int cap, int *count);

}  // namespace g6
