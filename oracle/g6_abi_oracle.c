/*
 * g6_abi_oracle.c -- the GRAPE-6 ABI (include/grape6.h:16-104) on the CPU,
 * over the oracle's FP64 restatement (oracle/g6_oracle.c).
 *
 * TEST INFRASTRUCTURE (the oracle).  The reference ships no GRAPE-6
 * emulator (only null stubs, src/node/dyn/hdyn/stubs/grape6_stubs.c);
 * oracle/build_ref.py links Starlab's own tools against this file
 * (kira_g6o, hsys_stats_g6o, get_densities_g6o) so that their GRAPE-6
 * branch (src/node/dyn/hdyn/evolve/hdyn_grape6.C) runs on the CPU with the
 * semantics the engine implements: j-memory by address with deferred
 * updates, prediction to ti, pair terms and nn of hdyn_ev.C:2019-2036 /
 * hdyn_inline.C:34-77, neighbour lists {j : dr.dr < h2_i} ascending with
 * self when npipes > 48 (hdyn_grape6.C:2309-2315), per-pipe capacity
 * G6ORACLE_NBMAX (default 4096) with the overflow conventions (read
 * returns 1; get returns 1 with *nblen = *max_length).  g6_npipes_() is
 * G6ORACLE_NPIPES (default 256).  One cluster (kira uses cluster_id 0).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void g6o_predict(int n, double ti, const double *tj, const double *x, const double *v, const double *a2,
                 const double *j6, double *xp, double *vp);
void g6o_force(int nj, const double *xj, const double *vj, const double *mj, const int *jindex, int ni,
               const int *index, const double *xi, const double *vi, double eps2, double *acc, double *jerk,
               double *pot, int *nn, double *nn_r2);
void g6o_neighbours(int nj, const double *xj, const int *jindex, int ni, const int *index, const double *xi,
                    const double *h2, int include_self, int *len, long long *off, int *nbl);

static int cap_j;
static double *X, *V, *A2, *J6, *M, *T, *XP, *VP;
static int *IDX;
static double ti_;
static int nj_, ni_;
static int *index_;
static double *xi_, *vi_, *h2_, eps2_;
static int *len_, *nbl_;
static long long *off_;
static int nb_ready_;

static void *grow(void *p, size_t bytes)
{
    void *q = realloc(p, bytes ? bytes : 1);
    if (!q) {
        fprintf(stderr, "g6 oracle: out of memory\n");
        exit(-1);
    }
    return q;
}

static int env_int(const char *name, int dflt)
{
    const char *s = getenv(name);
    return (s && *s) ? atoi(s) : dflt;
}

static void ensure_j(int n)
{
    if (n <= cap_j) return;
    int c = cap_j ? cap_j : 1024;
    while (c < n) c *= 2;
    size_t o = (size_t)cap_j, nn = (size_t)c;
    X = grow(X, 24 * nn); V = grow(V, 24 * nn); A2 = grow(A2, 24 * nn); J6 = grow(J6, 24 * nn);
    XP = grow(XP, 24 * nn); VP = grow(VP, 24 * nn);
    M = grow(M, 8 * nn); T = grow(T, 8 * nn); IDX = grow(IDX, 4 * nn);
    memset(X + 3 * o, 0, 24 * (nn - o)); memset(V + 3 * o, 0, 24 * (nn - o));
    memset(A2 + 3 * o, 0, 24 * (nn - o)); memset(J6 + 3 * o, 0, 24 * (nn - o));
    memset(M + o, 0, 8 * (nn - o)); memset(T + o, 0, 8 * (nn - o));
    for (size_t k = o; k < nn; k++) IDX[k] = -1;
    cap_j = c;
}

void g6_set_tunit_(int *u) { (void)u; }
void g6_set_xunit_(int *u) { (void)u; }
int g6_open_(int *id) { (void)id; return 0; }
int g6_close_(int *id) { (void)id; return 0; }

/* Calls of two i-particles sharing one index: the signature of kira's
 * binary perturbation call (hdyn_grape6.C:3415-3587 packs both components
 * with their top-level node's index).  Printed at exit with G6O_TRACE. */
static long long calls_, pair_calls_;

__attribute__((destructor)) static void trace_at_exit(void)
{
    if (getenv("G6O_TRACE")) fprintf(stderr, "g6 oracle trace: calls %lld pair_calls %lld\n", calls_, pair_calls_);
}
int g6_open_special(int ngpu, int *list) { (void)ngpu; (void)list; return 0; }
int g6_open_special2(int ngpu, int *list, int nmax) { (void)ngpu; (void)list; (void)nmax; return 0; }
int g6_reset_(int *id) { (void)id; return 0; }
int g6_reset_fofpga_(int *id) { (void)id; return 0; }
int g6_npipes_(void) { int n = env_int("G6ORACLE_NPIPES", 256); return n < 1 ? 1 : n; }
void g6_set_ti_(int *id, double *ti) { (void)id; ti_ = *ti; }
int g6_initialize_jp_buffer_(int *id, int *size) { (void)id; (void)size; return 0; }
int g6_flush_jp_buffer_(int *id) { (void)id; return 0; }

int g6_set_j_particle_(int *id, int *address, int *index, double *tj, double *dtj, double *mass, double k18[3],
                       double j6[3], double a2[3], double v[3], double x[3])
{
    (void)id; (void)dtj; (void)k18;
    int a = *address;
    if (a < 0) return -1;
    ensure_j(a + 1);
    memcpy(X + 3 * a, x, 24); memcpy(V + 3 * a, v, 24);
    memcpy(A2 + 3 * a, a2, 24); memcpy(J6 + 3 * a, j6, 24);
    M[a] = *mass;
    T[a] = *tj;
    IDX[a] = *index;
    return 0;
}

void g6calc_firsthalf_(int *id, int *nj, int *ni, int index[], double xi[][3], double vi[][3], double aold[][3],
                       double j6old[][3], double phiold[], double *eps2, double h2[])
{
    (void)id; (void)aold; (void)j6old; (void)phiold;
    nj_ = *nj;
    ni_ = *ni;
    calls_++;
    if (ni_ == 2 && index[0] == index[1]) pair_calls_++;
    ensure_j(nj_);
    index_ = grow(index_, 4 * (size_t)ni_);
    xi_ = grow(xi_, 24 * (size_t)ni_); vi_ = grow(vi_, 24 * (size_t)ni_); h2_ = grow(h2_, 8 * (size_t)ni_);
    memcpy(index_, index, 4 * (size_t)ni_);
    memcpy(xi_, xi, 24 * (size_t)ni_); memcpy(vi_, vi, 24 * (size_t)ni_);
    if (h2) memcpy(h2_, h2, 8 * (size_t)ni_); else memset(h2_, 0, 8 * (size_t)ni_);
    eps2_ = *eps2;
    nb_ready_ = 0;
    g6o_predict(nj_, ti_, T, X, V, A2, J6, XP, VP);
}

static void compute(double (*acc)[3], double (*jerk)[3], double *pot, int *nn)
{
    double *r2 = grow(NULL, 8 * (size_t)(ni_ > 0 ? ni_ : 1));
    int *nnb = nn ? nn : grow(NULL, 4 * (size_t)(ni_ > 0 ? ni_ : 1));
    g6o_force(nj_, XP, VP, M, IDX, ni_, index_, xi_, vi_, eps2_, &acc[0][0], &jerk[0][0], pot, nnb, r2);
    if (!nn) free(nnb);
    free(r2);
}

int g6calc_lasthalf_(int *id, int *nj, int *ni, int index[], double xi[][3], double vi[][3], double *eps2,
                     double h2[], double acc[][3], double jerk[][3], double pot[])
{
    (void)id; (void)nj; (void)ni; (void)index; (void)xi; (void)vi; (void)eps2; (void)h2;
    compute(acc, jerk, pot, NULL);
    return 0;
}

int g6calc_lasthalf2_(int *id, int *nj, int *ni, int index[], double xi[][3], double vi[][3], double *eps2,
                      double h2[], double acc[][3], double jerk[][3], double pot[], int nnbindex[])
{
    (void)id; (void)nj; (void)ni; (void)index; (void)xi; (void)vi; (void)eps2; (void)h2;
    compute(acc, jerk, pot, nnbindex);
    return 0;
}

int g6_read_neighbour_list_(int *id)
{
    (void)id;
    len_ = grow(len_, 4 * (size_t)(ni_ + 1));
    off_ = grow(off_, 8 * (size_t)(ni_ + 1));
    int self = g6_npipes_() > 48;
    g6o_neighbours(nj_, XP, IDX, ni_, index_, xi_, h2_, self, len_, off_, NULL);
    nbl_ = grow(nbl_, 4 * (size_t)(off_[ni_] + 1));
    g6o_neighbours(nj_, XP, IDX, ni_, index_, xi_, h2_, self, len_, off_, nbl_);
    nb_ready_ = 1;
    int cap = env_int("G6ORACLE_NBMAX", 4096);
    for (int i = 0; i < ni_; i++)
        if (len_[i] > cap) return 1;
    return 0;
}

int g6_read_neighbour_list_old_(int *id) { return g6_read_neighbour_list_(id); }

int g6_get_neighbour_list_(int *id, int *pipe, int *max_length, int *nblen, int nbl[])
{
    (void)id;
    if (!nb_ready_ || *pipe < 0 || *pipe >= ni_) {
        *nblen = 0;
        return -1;
    }
    int cap = env_int("G6ORACLE_NBMAX", 4096);
    int n = len_[*pipe];
    if (n > *max_length || n > cap) {
        int k = n < *max_length ? n : *max_length;
        memcpy(nbl, nbl_ + off_[*pipe], 4 * (size_t)k);
        *nblen = *max_length;
        return 1;
    }
    memcpy(nbl, nbl_ + off_[*pipe], 4 * (size_t)n);
    *nblen = n;
    return 0;
}
