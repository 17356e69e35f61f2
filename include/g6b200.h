/*
 * g6b200.h -- C ABI of the B200 GRAPE-6 force engine (libg6b200.so).
 *
 * The first block is the GRAPE-6 host-library ABI exactly as Starlab's
 * include/grape6.h:16-104 declares it and src/node/dyn/hdyn/evolve/
 * hdyn_grape6.C calls it: Fortran-style trailing underscores, every scalar by
 * pointer, `vec` arrays as double[][3] (include/starlab_vector.h: a vec is
 * three contiguous doubles).  Linking kira/hsys_stats/hscale against this
 * library ahead of the reference's null stubs
 * (src/node/dyn/hdyn/stubs/grape6_stubs.c) makes g6_npipes_() > 0, so kira
 * selects its GRAPE-6 code path (kira_config.C:62) unchanged.
 *
 * Semantics shared by all entry points:
 *   - cluster_id selects an independent engine instance (device-resident
 *     j-memory); kira always uses 0.  Instances open lazily.
 *   - int returns: 0 = OK.  g6calc_lasthalf*_ nonzero = engine error (kira
 *     then resets, reopens, reloads j and retries: hdyn_grape6.C:892-899).
 *   - j-particle updates are staged on the host and reach the device at the
 *     next g6calc_firsthalf_ / g6_flush_jp_buffer_.
 *   - g6calc_firsthalf_ starts the computation asynchronously; the matching
 *     g6calc_lasthalf*_ waits and writes the results.  Calls alternate.
 *   - The engine computes, for each i, the sum over j in [0, nj), j != the
 *     i's index, of the softened Newtonian pair terms (hdyn_ev.C:2019-2036):
 *     acc, full jerk, pot (< 0), plus the nearest neighbour address (r^2
 *     without softening, first address on ties) and, for h2[i] > 0, the
 *     neighbour list {j : |x_j - x_i|^2 < h2[i]}.
 *   - Precision mode per instance (g6b200_set_precision, or the environment
 *     variable G6B200_PRECISION=fp64|mixed read at open):
 *       G6B200_FP64  : FP64 prediction, differences, pair math, accumulation.
 *       G6B200_MIXED : FP64 prediction; positions as 47-bit fixed point held
 *                      in two FP32 words so x_j - x_i is exact before its one
 *                      rounding to FP32; FP32 pair math with a Newton-refined
 *                      rsqrt; FP32 partial sums over short j-chunks folded
 *                      into FP64 accumulators; particles whose sums are ill
 *                      conditioned (large, nearly cancelling terms: error
 *                      indicators accumulated by the kernel) recomputed in
 *                      FP64, so every particle meets acc, pot <= 1e-6 and
 *                      jerk <= 1e-5 relative to FP64.  Calls of fewer than
 *                      G6B200_MIXED_MIN_WORK (2^25) interactions run in
 *                      FP64 (they are latency-bound; kira's small blocks).
 */
#ifndef G6B200_H
#define G6B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GRAPE-6 ABI (include/grape6.h) ---------------------------------- */

/* grape6.h:18-19.  Fixed-point unit exponents of the GRAPE-6 hardware.
 * Accepted and ignored: this engine chooses its own scaling. */
void g6_set_tunit_(int *new_tunit);
void g6_set_xunit_(int *new_xunit);

/* grape6.h:21-22; called at hdyn_grape6.C:164,422,979.  Attach / detach the
 * engine (device buffers, stream).  Return 0. */
int g6_open_(int *cluster_id);
int g6_close_(int *cluster_id);

/* grape6.h:27-28 (sapporo extension; stub in
 * src/node/dyn/hdyn/stubs/sapporo_stubs.c:17-25 takes a third nmax arg).
 * Open cluster 0 on device list[0] (a one-GPU engine: entries past the first
 * are ignored); nmax is a j-capacity hint.  Return 0. */
int g6_open_special(int ngpu, int *list);
int g6_open_special2(int ngpu, int *list, int nmax);

/* grape6.h:32-33; hdyn_grape6.C:416-417.  Clear the engine's error state
 * and drop staged j updates; j-memory is kept (kira reloads it anyway). */
int g6_reset_(int *cluster_id);
int g6_reset_fofpga_(int *cluster_id);

/* grape6.h:36; kira_config.C:62,105.  Maximum ni per firsthalf call
 * (G6B200_NPIPES, default 256).  > 48 tells kira to use the GPU
 * conventions (self included in neighbour lists, hdyn_grape6.C:2309-2315). */
int g6_npipes_(void);

/* grape6.h:38; hdyn_grape6.C:516.  Block time the j-particles are
 * predicted to. */
void g6_set_ti_(int *cluster_id, double *ti);

/* grape6.h:39-49; hdyn_grape6.C:273-281.  Store j-particle `address`:
 * time tj, mass, k18 = k/18 (stored, unused by the 3rd-order predictor),
 * j6 = jerk/6, a2 = acc/2, velocity v and position x.  `index` is the id
 * compared against firsthalf's index[] to skip self-interaction; kira passes
 * index == address.  dtj is accepted and ignored.  Return 0, or -1 for a
 * negative address. */
int g6_set_j_particle_(int *cluster_id, int *address, int *index,
                       double *tj, double *dtj, double *mass,
                       double k18[3], double j6[3], double a2[3],
                       double v[3], double x[3]);

/* grape6.h:55-66; hdyn_grape6.C:675-677.  Start the force on ni (<= npipes)
 * i-particles from j-addresses [0, nj).  xi/vi are the i positions and
 * velocities (already predicted by the caller); aold/j6old/phiold are the
 * previous acc, full jerk and pot, accepted as scaling hints and unused;
 * *eps2 is the softening squared; h2[i] > 0 requests i's neighbour list. */
void g6calc_firsthalf_(int *cluster_id, int *nj, int *ni, int index[],
                       double xi[][3], double vi[][3], double aold[][3],
                       double j6old[][3], double phiold[], double *eps2,
                       double h2[]);

/* grape6.h:68-78.  Wait for the call started by firsthalf; write acc, full
 * jerk and pot.  Return 0 = OK. */
int g6calc_lasthalf_(int *cluster_id, int *nj, int *ni, int index[],
                     double xi[][3], double vi[][3], double *eps2,
                     double h2[], double acc[][3], double jerk[][3],
                     double pot[]);

/* grape6.h:80-92; hdyn_grape6.C:687-689.  As lasthalf, plus nnbindex[i],
 * the address of i's nearest neighbour (0 if it has none). */
int g6calc_lasthalf2_(int *cluster_id, int *nj, int *ni, int index[],
                      double xi[][3], double vi[][3], double *eps2,
                      double h2[], double acc[][3], double jerk[][3],
                      double pot[], int nnbindex[]);

/* grape6.h:94-95; hdyn_grape6.C:2062-2066.  Make the neighbour lists of the
 * last call readable.  Return 0 OK, 1 if some list exceeded the engine's
 * per-pipe capacity (G6B200_NBMAX, default 4096; kira then shrinks h2 and
 * retries), < 0 on error. */
int g6_read_neighbour_list_(int *cluster_id);
int g6_read_neighbour_list_old_(int *cluster_id);

/* grape6.h:97-101; hdyn_grape6.C:2302-2306.  Copy pipe's list (ascending
 * j-address) into nbl, at most *max_length entries; *nblen = its length.
 * Return 0, or 1 when the list is longer than *max_length or overflowed the
 * engine (then *nblen = *max_length, as the GRAPE-6 library does), -1 for a
 * bad pipe.  With npipes > 48 the list contains i itself. */
int g6_get_neighbour_list_(int *cluster_id, int *pipe, int *max_length,
                           int *nblen, int nbl[]);

/* grape6.h:104-105; hdyn_grape6.C:266-271,672-673.  DMA batching of j
 * writes: staging is always on, so initialize only sizes the staging buffer
 * and flush pushes staged updates to the device now. */
int g6_initialize_jp_buffer_(int *clusterid, int *size);
int g6_flush_jp_buffer_(int *clusterid);

/* Named in the engine's specification but absent from grape6.h (the
 * reference passes the sphere per i through firsthalf's h2[]).  Sets a
 * default h2 used for every i when a caller passes h2 == NULL. */
void g6_set_neighbour_list_sphere_(int *cluster_id, double *h2);

/* ---- Extensions (no counterpart in grape6.h) ------------------------- */

enum { G6B200_FP64 = 0, G6B200_MIXED = 1 };

/* Select the precision mode of an instance (opens it if needed). */
int g6b200_set_precision(int cluster_id, int mode);
int g6b200_get_precision(int cluster_id);

/* Maximum ni per firsthalf for this instance (default G6B200_NPIPES or
 * 256).  g6_npipes_() reports cluster 0's value. */
int g6b200_set_npipes(int cluster_id, int npipes);
int g6b200_get_npipes(int cluster_id);

/* Pin the force kernel's launch shape (used by the autotuner and the
 * benchmarks): il i-lanes per warp (1, 8, 32), r i-particles per thread
 * (1, or 2 or 4 with il = 32; 4 is mixed mode only), warps per CTA (power of two <= 8), h warps
 * splitting each CTA's j-tile, nsplit CTAs along j.  il = 0 returns to the
 * built-in heuristic.  g6b200_get_config reports the shape of the last call
 * as {il, r, warps, h, nsplit}. */
int g6b200_set_config(int cluster_id, int il, int r, int warps, int h, int nsplit);
int g6b200_get_config(int cluster_id, int *out5);

/* Upload n j-particles in one call (SoA-free batched form of
 * g6_set_j_particle_: arrays of n entries, vectors as [n][3]). */
int g6b200_set_j_particles(int cluster_id, int n, const int *address,
                           const int *index, const double *tj,
                           const double *mass, const double (*k18)[3],
                           const double (*j6)[3], const double (*a2)[3],
                           const double (*v)[3], const double (*x)[3]);

/* Self-gravity sweep (blocking): acc, full jerk, pot and nn of the stored
 * j-particles at addresses [i0, i0+ni) themselves, from all j in [0, nj),
 * each i predicted to the current ti on the device like the j-side -- the
 * all-particle pass of an energy evaluation (hdyn_grape6.C:1254-1305) or of
 * a shared-timestep step, without host i-arrays.  With all four output
 * pointers NULL the results stay in device memory (timing runs). */
int g6b200_sweep(int cluster_id, int nj, int i0, int ni, double eps2,
                 double (*acc)[3], double (*jerk)[3], double *pot, int *nn);

/* Counters since open: calls, interactions, j updates, bytes moved, kernel
 * launches, and device times (CUDA events on the instance's stream) of the
 * last call: force kernel (+ split reduction), predictor (0 if the cached
 * prediction was reused), whole call. */
typedef struct {
    long long calls;
    long long interactions;
    long long j_updates;
    long long h2d_bytes;
    long long d2h_bytes;
    double last_force_ms;
    double last_predict_ms;
    double last_call_ms;
    long long launches;
    long long refined;  /* mixed mode: particles recomputed in FP64 (ill-conditioned sums) */
} g6b200_stats;
int g6b200_get_stats(int cluster_id, g6b200_stats *out);

/* ---- Ensemble of independent clusters (no counterpart in grape6.h) ----
 *
 * Many clusters integrated together on one GPU with kira's scheme for its
 * top-level nodes: 4th-order Hermite predictor/corrector (include/_dyn_.h:
 * 265-299, hdyn_ev.C:1717-1718), individual power-of-two block steps from an
 * Aarseth-type criterion with accuracy eta, first steps from 0.01|a|/|j|,
 * steps capped at 1/16.  State stays on the device; every iteration advances
 * each unfinished cluster by its own next block, and the force work of all
 * clusters runs as one persistent launch over a (cluster, i-tile, j-split)
 * work list (graph-captured).  A cluster's sums depend on that cluster alone,
 * so its trajectory is bit-identical whether it is integrated alone or with
 * others (same i-tile shape).  run with per_cluster = 1 instead drives the
 * same integration through one plain engine call per cluster per block
 * (host prediction and correction), the baseline the batched path is
 * measured against. */
typedef struct g6b200_ensemble g6b200_ensemble;
typedef struct {
    double seconds;
    long long interactions;
    long long iterations;
    long long launches;
    int tuned_h;
    int tuned_tasks;     /* j-split factor chosen by the tuner (tasks wanted per cluster) */
    long long lane_interactions; /* i-lanes x j-records the force kernel ran (whole i-tiles,
                                  * j padded to its tile): interactions / lane_interactions is
                                  * the share of the kernel's lanes doing useful pairs */
} g6b200_ens_stats;
g6b200_ensemble *g6b200_ens_create(int nclusters, const int *n, const double *eps2, double eta,
                                   int precision, int device);
int g6b200_ens_set_cluster(g6b200_ensemble *h, int c, const double *m, const double (*x)[3],
                           const double (*v)[3]);
/* Forces and first steps at t = 0 (after every cluster has been set). */
int g6b200_ens_start(g6b200_ensemble *h);
/* Advance every cluster to t_end (a multiple of 1/16, so all particles land
 * on it exactly).  tune = 1 first times the i-tile shapes on live
 * iterations and keeps the fastest. */
int g6b200_ens_run(g6b200_ensemble *h, double t_end, int per_cluster, int tune, g6b200_ens_stats *out);
/* Kinetic and potential energy of every cluster ([2*nclusters]: ek, ep);
 * valid when all particles share one time (start, or after a run). */
int g6b200_ens_energies(g6b200_ensemble *h, double *ek_ep);
/* State of cluster c (any pointer may be NULL): masses, positions,
 * velocities, acc, jerk, times and current steps of its particles. */
int g6b200_ens_get_cluster(g6b200_ensemble *h, int c, double *m, double (*x)[3], double (*v)[3],
                           double (*acc)[3], double (*jerk)[3], double *t, double *dt);
void g6b200_ens_destroy(g6b200_ensemble *h);

/* ---- Force-call server with continuous batching (no counterpart) -----
 *
 * Clients on any host threads open clusters (device-resident j-memory,
 * admitted against an HBM budget: g6b200_srv_open_cluster blocks until the
 * cluster's footprint fits), load j-particles, then submit force calls -- a
 * block time, nj and an i-block with predicted positions and velocities, the
 * content of one g6calc_firsthalf_ -- and wait for acc, jerk, pot and nn (the
 * outputs of g6calc_lasthalf2_).  Two dispatcher threads (lanes) run the
 * pending calls as batched launches: calls with ni*nj up to G6B200_SRV_SMALL
 * (default 1e8 pair interactions) as one persistent launch on a
 * high-priority stream, larger calls one CTA per task on a low-priority
 * stream, so short calls are not held behind long ones; calls arriving while
 * a launch runs join the next one.  Every call predicts its cluster's
 * j-set into its own buffer, so calls of one cluster at different block times
 * may share a launch.  A call sees the j-particles loaded before its launch is
 * dispatched, so a client that updates j-particles between calls (as kira
 * does after each block) waits for a call before loading the next updates.
 * A call's results do not depend on which other calls
 * share its launch (bit-identical alone or mixed).  precision: G6B200_FP64 or
 * G6B200_MIXED.  No neighbour lists on this path. */
typedef struct g6b200_server g6b200_server;
typedef struct {
    long long batches, requests, interactions, max_batch;
    double gpu_ms;    /* device time of all batches */
    double batch_ms;  /* host wall time spent running batches */
    double queue_ms;  /* summed time calls waited before their batch began */
} g6b200_srv_stats_t;
g6b200_server *g6b200_srv_create(int device, long long hbm_budget_bytes, int precision, int max_batch);
int g6b200_srv_open_cluster(g6b200_server *h, long long n_cap, double eps2);  /* cluster id or < 0 */
int g6b200_srv_close_cluster(g6b200_server *h, int cluster);
/* Load n j-particles at addresses address[k] (NULL: 0..n-1), as
 * g6_set_j_particle_ (a2 = acc/2, j6 = jerk/6). */
int g6b200_srv_set_j(g6b200_server *h, int cluster, int n, const int *address, const double *tj,
                     const double *mass, const double (*j6)[3], const double (*a2)[3],
                     const double (*v)[3], const double (*x)[3]);
long long g6b200_srv_submit(g6b200_server *h, int cluster, double ti, int nj, int ni, const int *index,
                            const double (*xi)[3], const double (*vi)[3]);  /* request id or < 0 */
/* Block until the request is done; outputs as g6calc_lasthalf2_; latency_s
 * = time from submit to completion. */
int g6b200_srv_wait(g6b200_server *h, long long request, double (*acc)[3], double (*jerk)[3], double *pot,
                    int *nn, double *latency_s);
/* As g6b200_srv_wait, plus the sequence number of the batch that ran the
 * call and how many calls that batch held (the calls that shared its
 * launch). */
int g6b200_srv_wait_batch(g6b200_server *h, long long request, double (*acc)[3], double (*jerk)[3], double *pot,
                          int *nn, double *latency_s, long long *batch, int *batch_size);
/* hold != 0: the dispatchers take no new calls; hold = 0: every call
 * pending then goes into the next batch of its lane (up to max_batch)
 * together -- a burst gathered on purpose. */
void g6b200_srv_hold(g6b200_server *h, int hold);
int g6b200_srv_stats(g6b200_server *h, g6b200_srv_stats_t *out);
void g6b200_srv_destroy(g6b200_server *h);

/* Potential only.  The reference computes energies through the full pair
 * call: grape6_calculate_energies (src/node/dyn/hdyn/evolve/
 * hdyn_grape6.C:1403-1546) drives force_by_grape(..., pot_only = true)
 * (:474-910), which sends time 0 and unpredicted positions and reads back
 * only pot; the ABI has no way to say so, so acc, jerk and nn are computed
 * and discarded.  This extension runs a potential-only kernel: pot[ni] of
 * the i-particles (index and xi as in g6calc_firsthalf_) from the j-memory
 * predicted to the current ti.  ni <= npipes.  Blocking.  0 = OK. */
int g6b200_calc_pot(int cluster_id, int nj, int ni, const int *index, const double (*xi)[3], double eps2,
                    double *pot);
/* Energies of the stored particles [0, nj) among themselves at the current
 * ti (set ti and tj to 0 for unpredicted positions, as the reference's
 * energy call does): epot = 1/2 sum m_i pot_i, ekin = 1/2 sum m_i |v_i|^2,
 * both formed on the device in FP64 in a fixed order; pot [nj] is filled
 * when not NULL.  The potential-only counterpart of the energy sums
 * grape6_calculate_energies forms on the host (hdyn_grape6.C:1512-1527).
 * Blocking.  0 = OK. */
int g6b200_energies(int cluster_id, int nj, double eps2, double *epot, double *ekin, double *pot);

/* One cluster's j-set split across GPUs, one process per GPU.  Counterpart
 * of the reference's MPI force (src/node/dyn/hdyn/evolve/kira_ev.C:275-420:
 * each rank sums over its range of j, then MPI_Allreduce SUM of acc/jerk/pot
 * at :327-328 and MINLOC of the nearest neighbour at :409-410).  Here the
 * global j-set is cut into blocks of block_j j (a multiple of 256); each
 * rank holds a contiguous run of whole blocks at local addresses 0..nj-1,
 * starting at global address j_offset.  Each block's FP64 partial sums are
 * converted to 64-bit fixed point on a per-(i, quantity) scale all ranks
 * agree on and summed exactly, so the results are bit-identical for any
 * number of ranks.  The caller runs the collectives on its own stream
 * `stream` (a cudaStream_t of this instance's device) over int64 device
 * buffers: agree [8 ni], sums [7 ni], negj [ni].
 *   1. g6b200_split_begin: i-block as in g6calc_firsthalf_ (index = the
 *      i's LOCAL address, or one no local j has); returns when agree is
 *      written.  Then all_reduce(agree, MAX).
 *   2. g6b200_split_fix: nblocks_total = global block count.  Then
 *      all_reduce(sums, SUM) and all_reduce(negj, MAX).
 *   3. g6b200_split_finish: acc, jerk, pot, nn (GLOBAL address, 0 if none,
 *      as g6calc_lasthalf2_) into host arrays; blocking.
 * No other call on the instance between begin and finish.  In the mixed
 * mode the ranks' fixed-point position grids must agree: every rank calls
 * g6b200_set_position_range with the same bound on |x| first.  Returns 0 =
 * OK. */
int g6b200_split_begin(int cluster_id, int nj, int ni, const int *index, const double (*xi)[3],
                       const double (*vi)[3], double eps2, int block_j, long long *agree, void *stream);
int g6b200_split_fix(int cluster_id, long long nblocks_total, long long j_offset, const long long *agree,
                     long long *sums, long long *negj, void *stream);
int g6b200_split_finish(int cluster_id, long long nblocks_total, long long nj_total, const long long *agree,
                        const long long *sums, const long long *negj, void *stream, double (*acc)[3],
                        double (*jerk)[3], double *pot, int *nn);
int g6b200_set_position_range(int cluster_id, double xmax);

/* Device-resident serving of many clusters' force calls (no counterpart in
 * the reference, whose unit of work is one force_by_grape call,
 * src/node/dyn/hdyn/evolve/hdyn_grape6.C:474-910).  One persistent
 * cooperative kernel polls a ring of requests in pinned host memory,
 * gathers every pending call into one batch (prediction of each call's
 * j-set to its block time, one (call, i-tile, j-split) task list, results
 * written back into the request's pinned buffer) and marks them done: no
 * launch per call or per batch.  Every wait in the kernel is bounded by the
 * global timer: it leaves after G6B200_RES_IDLE_MS (20) ms without calls and
 * is launched again by the next submit; a grid barrier that does not
 * complete within G6B200_RES_WAIT_MS (2000) ms ends it with an error and the
 * calls it held fail with code 2.  Clusters are admitted against an HBM
 * budget (open blocks until the footprint fits).  set_j waits until no call
 * of the cluster is in flight and copies the touched j rows with the copy
 * engine.  A call sees the j-particles set before it was submitted; its
 * results are bit-identical alone and in any mix.  wait returns 0, 2 (the
 * kernel left before the call completed, or could not be launched for it),
 * 3 (a j-tile copy wait timed out),
 * 4 (positions outside the fixed-point range: the range is widened, submit
 * again), < 0 (bad request).  hold(1) keeps calls from the kernel until
 * hold(0) releases them together.  selftest_stall makes the kernel's CTA 0
 * leave once without arriving at a barrier (the others' bounded waits run
 * out: the failure path of the loop, without a GPU fault). */
typedef struct g6b200_resident g6b200_resident;
typedef struct {
    long long batches, calls, launches, recoveries;
    int max_batch;
} g6b200_res_stats_t;
g6b200_resident *g6b200_res_create(int device, long long hbm_budget_bytes, int precision, int max_batch);
int g6b200_res_open_cluster(g6b200_resident *h, long long n_cap, double eps2);  /* cluster id or < 0 */
int g6b200_res_close_cluster(g6b200_resident *h, int cluster);
int g6b200_res_set_j(g6b200_resident *h, int cluster, int n, const int *address, const double *tj,
                     const double *mass, const double (*j6)[3], const double (*a2)[3], const double (*v)[3],
                     const double (*x)[3]);
long long g6b200_res_submit(g6b200_resident *h, int cluster, double ti, int nj, int ni, const int *index,
                            const double (*xi)[3], const double (*vi)[3]);  /* request id or < 0 */
int g6b200_res_wait(g6b200_resident *h, long long request, double (*acc)[3], double (*jerk)[3], double *pot,
                    int *nn, double *latency_s, long long *batch, int *batch_size);
void g6b200_res_hold(g6b200_resident *h, int hold);
void g6b200_res_selftest_stall(g6b200_resident *h);
int g6b200_res_stats(g6b200_resident *h, g6b200_res_stats_t *out);
void g6b200_res_destroy(g6b200_resident *h);

/* The FP32 FLOP rate this GPU sustains (no counterpart in the reference):
 * a kernel of independent packed FP32x2 FMA chains on every SM, timed with
 * CUDA events -- the measured denominator of the force kernel's roofline.
 * Writes TFLOP/s; returns 0, or -1 on a CUDA error. */
int g6b200_measure_fp32_peak(int device, double *tflops);

/* Self-test of failure detection (no counterpart in the reference).  Every
 * j-tile copy the force kernel waits for is waited on with a time bound;
 * when a bound runs out the kernel sets a status bit and returns, and
 * g6calc_lasthalf2_ returns 3 (kira then resets and retries).  This runs
 * that bounded wait on a barrier nothing arrives at, through the same status
 * word and host path: it returns 3 after about limit_ms (1 ms if <= 0), with
 * the message in g6b200_last_error(), and the instance stays usable.  -1 on
 * a CUDA error or while a firsthalf call is pending. */
int g6b200_selftest_copy_timeout(int cluster_id, double limit_ms);

/* Allocation-free force evaluation.  No counterpart in the reference: the
 * GRAPE-6 library owned its board memory, and this entry point exists for
 * callers of this library that cannot call cudaMalloc -- a host program
 * whose own allocator or fixed memory budget owns the device, a loop that
 * must not pay the device-wide synchronisation of cudaMalloc/cudaFree, a
 * plug-in that is handed only buffers it does not own.  The caller passes
 * DEVICE pointers for all inputs and outputs: xj, vj [nj][3] and mj [nj]
 * (positions/velocities already at the block time; no prediction is done),
 * index_i [ni] (the j-address of each i, skipped in its sum; may be NULL),
 * xi, vi [ni][3], and outputs acc, jerk [ni][3], pot [ni], nn [ni].  The
 * sums are FP64 (as G6B200_FP64).  The j-split partial sums use one static
 * device array of G6B200_NOALLOC_MAX_NI records (80 B each, 2.5 MiB), which
 * every GPU that loads the library holds until exit; ni beyond
 * G6B200_NOALLOC_MAX_NI is rejected (returns -1, message in
 * g6b200_last_error()).  Work is queued on `stream` (a cudaStream_t, NULL =
 * the legacy default stream) and the call returns without waiting.  The
 * first call on a device looks up the array's device address there (with
 * that device current) and should come before any stream capture.  Calls
 * share the array: two calls whose kernels overlap on the GPU race and give
 * wrong results; order them on one stream.  A CUDA error already pending on
 * the calling thread (left by earlier work) is reported as such with -3 and
 * nothing is launched.  Returns 0, -1 (size beyond the limit), -2 (bad
 * argument), -3 (CUDA error). */
#define G6B200_NOALLOC_MAX_NI 32768
int g6b200_force_noalloc(int nj, const double *xj, const double *vj,
                         const double *mj, int ni, const int *index_i,
                         const double *xi, const double *vi, double eps2,
                         double *acc, double *jerk, double *pot, int *nn,
                         void *stream);

/* Message of the last error on this thread ("" if none). */
const char *g6b200_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* G6B200_H */
