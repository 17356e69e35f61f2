/*
 * h3b200.h -- C ABI of the B200 GRAPE-4 (HARP-3) force engine (libh3b200.so).
 *
 * The GRAPE-4 host-library ABI as Starlab's include/grape4.h:22-45 declares
 * it and src/node/dyn/hdyn/evolve/hdyn_grape4.C calls it (kira's
 * config == 1 branch, selected when h3npipe_() > 0: kira_config.C:65,95).
 * Fortran-style trailing underscores, scalars by pointer, `vec` arrays as
 * double[][3] (include/starlab_vector.h).  The semantics are those of the
 * reference's IEEE GRAPE-4 simulator, src/harpsims/harp3fastsim.c, the only
 * executable definition of the ABI in the reference tree.
 *
 * This is a separate library from libg6b200.so on purpose: kira adds 1 for a
 * GRAPE-4 and 2 for a GRAPE-6 to its configuration and takes the GRAPE-4
 * branch whenever the sum is odd (kira_config.C:65-95), so one library that
 * answered both h3npipe_() and g6_npipes_() would turn every GRAPE-6 caller
 * into a GRAPE-4 one.  Link libh3b200.so ahead of the reference's null stubs
 * (src/node/dyn/hdyn/stubs/grape4_stubs.c) to accelerate the GRAPE-4 branch.
 *
 * Pipeline (harp3fastsim.c:223-321), FP64 throughout:
 *   prediction of every j in [0, nj) to ti with s = ti - tj:
 *     xp = ((jj s + aj) s + v) s + x,   vp = (1.5 jj s + aj) 2 s + v,
 *     where aj = acc/2 and jj = jerk/6 as the caller stores them
 *     (hdyn_grape4.C:265-266);
 *   for each i: r2 = 2 eps2[i] + |xp_j - x_i|^2; pairs with r2 > 0 add
 *     acc += m r^-3 dr,  jerk += m r^-3 (dv - 3 (dr.dv)/r2 dr),
 *     pot -= m / r
 *     (no exclusion by index: kira stores the current block at the block
 *     time, so a particle meets itself at r2 == 0 when eps2 == 0);
 *   neighbour list of i: every j with r2 < 2 h2[i], ascending address.
 * The factor 2 on eps2 and h2 is the simulator's (harp3fastsim.c:240-242,
 * "to mimic HARP chips").  The simulator leaves pot at 0; this engine returns
 * the potential, which kira's GRAPE-4 energy path reads
 * (grape4_calculate_energies, hdyn_grape4.C:789-840: epot = sum m pot / 2).
 *
 * Error behaviour follows the simulator, whose entry points return nothing:
 * ni above h3npipe_(), nj above h3jpmax_() in one DMA, or an engine failure
 * print a message on stderr and exit(-1) (harp3fastsim.c:155-158,
 * 232-236, 329-333).
 *
 * Environment: G6B200_DEVICE (GPU ordinal, default 0), H3B200_NPIPES
 * (h3npipe_(), default 4096), G6B200_NBMAX (per-i list capacity of the force
 * pass; longer lists are recomputed for their pipe, so h3nblist_ never
 * truncates).
 */
#ifndef H3B200_H
#define H3B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* grape4.h:22-23; hdyn_grape4.C:800,1151,520.  Attach / detach the engine. */
void h3open_(void);
void h3close_(void);

/* grape4.h:24; kira_config.C:65, hdyn_grape4.C:319.  i-slots per call
 * (H3B200_NPIPES, default 4096).  Consecutive slots with identical inputs
 * (kira's padding with copies of the last i, and the slot pairs of a build
 * with USE_HALF_CHIP, hdyn_grape4.C:350-382) are computed once. */
int h3npipe_(void);

/* grape4.h:25-26; hdyn_grape4.C:419.  Boards: always 1. */
void h3setnboards_(int *nboards);
int h3getnboards_(void);

/* grape4.h:27; hdyn_grape4.C:290-291,390.  Returns 0: firsthalf is
 * asynchronous and lasthalf waits for it. */
unsigned int h3wait_(void);

/* grape4.h:28; hdyn_grape4.C:347.  Time the j-particles are predicted to. */
void h3setti_(double *ti);

/* grape4.h:29-30.  Hardware mode and LED controls: accepted, no effect. */
void h3setmode_(int *mode, int *iboard);
void h3setled_(int *mode, int *iboard);

/* grape4.h:31; hdyn_grape4.C:252.  Largest nj of one DMA (1048576). */
int h3jpmax_(void);

/* grape4.h:32 (harp3fastsim.c:122-137): h3mjpdma_indirect_ into buffer 0
 * followed by h3mjpdma_start_ of it. */
void h3jpdma_indirect_(int *nj, int *hostindex, double xj[][3], double vj[][3], double aj[][3],
                       double jj[][3], double *mj, double *tj, int *mode);

/* grape4.h:33; hdyn_grape4.C:285-286 (harp3fastsim.c:140-180).  Copy
 * nj j-particles into DMA buffer *buff_id (the next unused one when
 * negative): entry i is host element hostindex[i] - 1 of each array and goes
 * to j-address hostindex[i] - 1.  aj = acc/2, jj = jerk/6.  `mode` is
 * accepted and ignored, as the simulator does.  Buffers 0..63. */
void h3mjpdma_indirect_(int *nj, int *hostindex, double xj[][3], double vj[][3], double aj[][3],
                        double jj[][3], double *mj, double *tj, int *mode, int *buff_id);

/* grape4.h:34; hdyn_grape4.C:287 (harp3fastsim.c:182-206).  Commit DMA
 * buffer *buff_id to j-memory (it reaches the device at the next calc). */
void h3mjpdma_start_(int *buff_id);

/* grape4.h:35 (harp3fastsim.c:208-215, there named h3jpdma_flush_).
 * Commit every buffer filled with a negative buff_id, then forget them. */
void h3mjpdma_flush_(void);

/* grape4.h:36-37 (harp3fastsim.c:400-414).  firsthalf + lasthalf. */
void h3calc_(int *nj, int *ni, double xi[][3], double vi[][3], double *eps2, double *h2,
             double acc[][3], double jerk[][3], double *pot);

/* grape4.h:38; hdyn_grape4.C:389 (harp3fastsim.c:223-266).  Start the
 * forces on ni i-slots from j-addresses [0, nj); eps2[i] and h2[i] per slot. */
void h3calc_firsthalf_(int *nj, int *ni, double xi[][3], double vi[][3], double *eps2, double *h2);

/* grape4.h:39; hdyn_grape4.C:391 (harp3fastsim.c:268-335).  Wait, write
 * acc, jerk and pot of the first ni slots. */
void h3calc_lasthalf_(int *ni, double acc[][3], double jerk[][3], double *pot);

/* grape4.h:40; hdyn_grape4.C:420.  Make the last call's neighbour lists
 * readable. */
void h3nbread_(int *nboards);

/* grape4.h:41; hdyn_grape4.C:867 (harp3fastsim.c:440-451).  Copy the list of
 * i-slot *chip (ascending j-address) into nblist and return its length.
 * nblist must hold that many entries (kira's holds every j). */
int h3nblist_(int *board, int *chip, int *nblist);

/* grape4.h:42.  Length of i-slot chip's list. */
int count_nblist_low(int board, int chip);

/* grape4.h:43-45.  Debug level, DMA buffer check, time-check mode: accepted,
 * no effect. */
void h3setdebuglevel_(int *debug_level);
void h3checkdmabuffers_(void);
void set_time_check_mode(int mode);

/* Simulator entry points outside grape4.h (harp3fastsim.c:208-220). */
void h3jpdma_flush_(void);
void h3jpdma_reset_(void);

/* ---- Extensions (no counterpart in grape4.h) ------------------------- */

/* Text of the last error of this library (empty if none). */
const char *h3b200_last_error(void);

/* Counters of the engine behind the ABI. */
typedef struct {
    long long calls;        /* force calls launched */
    long long slots;        /* i-slots requested (sum of ni) */
    long long computed;     /* distinct i computed after slot deduplication */
    long long interactions; /* computed i x nj */
    long long j_updates;    /* j-particles committed */
    long long launches;     /* kernels launched */
} h3b200_stats;
int h3b200_get_stats(h3b200_stats *out);

#ifdef __cplusplus
}
#endif

#endif /* H3B200_H */
