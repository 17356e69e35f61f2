/*
 * h3_oracle.c -- the GRAPE-4 ABI (include/grape4.h:22-45) on the CPU, over
 * the oracle's restatement of the reference simulator's pipeline
 * (oracle/g4_oracle.c).
 *
 * TEST INFRASTRUCTURE (the oracle).  oracle/build_ref.py links Starlab's own
 * kira and hsys_stats against it (kira_g4o, hsys_stats_g4o) so that the
 * reference's GRAPE-4 branch (src/node/dyn/hdyn/evolve/hdyn_grape4.C) can
 * be run on the CPU with a pipeline that, unlike the simulator
 * (src/harpsims/harp3fastsim.c: 1000 j, 3 pipes, pot left at 0), has no
 * static limits and returns the potential.  The GPU library is compared
 * with these runs; nothing of the engine links this file.
 *
 * ABI behaviour as in the simulator: DMA buffers (indirect gather at
 * hostindex - 1, commit on start, :140-206), prediction at firsthalf
 * (:223-266), the pair loop at lasthalf (:268-335), neighbour lists per
 * slot (:440-451).  h3npipe_() is H3ORACLE_NPIPES (default 64).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void g4o_predict(int n, double ti, const double *tj, const double *x, const double *v, const double *aj,
                 const double *jj, double *xp, double *vp);
void g4o_force(int nj, const double *xj, const double *vj, const double *mj, int ni, const double *xi,
               const double *vi, const double *eps2, const double *h2, double *acc, double *jerk,
               double *pot, int *nbcount, int *nblist, int nbcap);

#define NBUF 64

typedef struct { int addr; double x[3], v[3], a[3], j[3], m, t; } jent;

static int cap_j;
static double *X, *V, *A, *J, *M, *T, *XP, *VP;
static jent *buf[NBUF];
static int buf_n[NBUF], buf_cap[NBUF], buff_used;
static double ti_;
static int nj_, ni_, nb_cap_;
static double *xi_, *vi_, *e_, *h_;
static int *cnt_, *lists_;

static void *grow(void *p, size_t bytes)
{
    void *q = realloc(p, bytes ? bytes : 1);
    if (!q) {
        fprintf(stderr, "h3 oracle: out of memory\n");
        exit(-1);
    }
    return q;
}

static void ensure_j(int n)
{
    if (n <= cap_j) return;
    int c = cap_j ? cap_j : 1024;
    while (c < n) c *= 2;
    size_t o = (size_t)cap_j, nn = (size_t)c;
    X = grow(X, 24 * nn); V = grow(V, 24 * nn); A = grow(A, 24 * nn); J = grow(J, 24 * nn);
    M = grow(M, 8 * nn); T = grow(T, 8 * nn); XP = grow(XP, 24 * nn); VP = grow(VP, 24 * nn);
    memset(X + 3 * o, 0, 24 * (nn - o)); memset(V + 3 * o, 0, 24 * (nn - o));
    memset(A + 3 * o, 0, 24 * (nn - o)); memset(J + 3 * o, 0, 24 * (nn - o));
    memset(M + o, 0, 8 * (nn - o)); memset(T + o, 0, 8 * (nn - o));
    cap_j = c;
}

int h3npipe_(void)
{
    const char *s = getenv("H3ORACLE_NPIPES");
    int n = (s && *s) ? atoi(s) : 64;
    return n < 1 ? 1 : n;
}

void h3open_(void) {}
void h3close_(void) {}
void h3setnboards_(int *n) { (void)n; }
int h3getnboards_(void) { return 1; }
unsigned int h3wait_(void) { return 0; }
void h3setti_(double *ti) { ti_ = *ti; }
void h3setmode_(int *a, int *b) { (void)a; (void)b; }
void h3setled_(int *a, int *b) { (void)a; (void)b; }
int h3jpmax_(void) { return 1 << 20; }
void h3setdebuglevel_(int *l) { (void)l; }
void h3checkdmabuffers_(void) {}
void set_time_check_mode(int m) { (void)m; }

void h3mjpdma_indirect_(int *nj, int *hostindex, double (*xj)[3], double (*vj)[3], double (*aj)[3],
                        double (*jj)[3], double *mj, double *tj, int *mode, int *buff_id)
{
    (void)mode;
    int b = (buff_id && *buff_id >= 0) ? *buff_id : buff_used++;
    if (b < 0 || b >= NBUF) {
        fprintf(stderr, "h3 oracle: DMA buffer %d out of range\n", b);
        exit(-1);
    }
    if (*nj > buf_cap[b]) {
        buf[b] = grow(buf[b], sizeof(jent) * (size_t)*nj);
        buf_cap[b] = *nj;
    }
    for (int i = 0; i < *nj; i++) {
        int h = hostindex[i] - 1;
        jent *q = &buf[b][i];
        q->addr = h;
        memcpy(q->x, xj[h], 24); memcpy(q->v, vj[h], 24);
        memcpy(q->a, aj[h], 24); memcpy(q->j, jj[h], 24);
        q->m = mj[h];
        q->t = tj[h];
    }
    buf_n[b] = *nj;
}

void h3mjpdma_start_(int *buff_id)
{
    int b = *buff_id;
    for (int i = 0; i < buf_n[b]; i++) {
        jent *q = &buf[b][i];
        ensure_j(q->addr + 1);
        memcpy(X + 3 * q->addr, q->x, 24); memcpy(V + 3 * q->addr, q->v, 24);
        memcpy(A + 3 * q->addr, q->a, 24); memcpy(J + 3 * q->addr, q->j, 24);
        M[q->addr] = q->m;
        T[q->addr] = q->t;
    }
}

void h3jpdma_indirect_(int *nj, int *hostindex, double (*xj)[3], double (*vj)[3], double (*aj)[3],
                       double (*jj)[3], double *mj, double *tj, int *mode)
{
    int zero = 0;
    h3mjpdma_indirect_(nj, hostindex, xj, vj, aj, jj, mj, tj, mode, &zero);
    h3mjpdma_start_(&zero);
}

void h3mjpdma_flush_(void)
{
    for (int b = 0; b < buff_used && b < NBUF; b++) h3mjpdma_start_(&b);
    buff_used = 0;
}

void h3jpdma_flush_(void) { h3mjpdma_flush_(); }
void h3jpdma_reset_(void) { buff_used = 0; }

void h3calc_firsthalf_(int *nj, int *ni, double (*xi)[3], double (*vi)[3], double *eps2, double *h2)
{
    nj_ = *nj;
    ni_ = *ni;
    ensure_j(nj_);
    xi_ = grow(xi_, 24 * (size_t)ni_); vi_ = grow(vi_, 24 * (size_t)ni_);
    e_ = grow(e_, 8 * (size_t)ni_); h_ = grow(h_, 8 * (size_t)ni_);
    memcpy(xi_, xi, 24 * (size_t)ni_); memcpy(vi_, vi, 24 * (size_t)ni_);
    memcpy(e_, eps2, 8 * (size_t)ni_); memcpy(h_, h2, 8 * (size_t)ni_);
    g4o_predict(nj_, ti_, T, X, V, A, J, XP, VP);
}

void h3calc_lasthalf_(int *ni, double (*acc)[3], double (*jerk)[3], double *pot)
{
    (void)ni;
    /* every list fits: capacity nj */
    nb_cap_ = nj_ > 0 ? nj_ : 1;
    cnt_ = grow(cnt_, 4 * (size_t)ni_);
    lists_ = grow(lists_, 4 * (size_t)ni_ * nb_cap_);
    g4o_force(nj_, XP, VP, M, ni_, xi_, vi_, e_, h_, &acc[0][0], &jerk[0][0], pot, cnt_, lists_, nb_cap_);
}

void h3calc_(int *nj, int *ni, double (*xi)[3], double (*vi)[3], double *eps2, double *h2, double (*acc)[3],
             double (*jerk)[3], double *pot)
{
    h3calc_firsthalf_(nj, ni, xi, vi, eps2, h2);
    h3calc_lasthalf_(ni, acc, jerk, pot);
}

void h3nbread_(int *n) { (void)n; }

int h3nblist_(int *board, int *chip, int *nblist)
{
    (void)board;
    if (*chip < 0 || *chip >= ni_) return 0;
    int n = cnt_[*chip];
    memcpy(nblist, lists_ + (size_t)*chip * nb_cap_, 4 * (size_t)n);
    return n;
}

int count_nblist_low(int board, int chip)
{
    (void)board;
    return (chip < 0 || chip >= ni_) ? 0 : cnt_[chip];
}
