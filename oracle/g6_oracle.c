/*
 * g6_oracle.c -- FP64 CPU restatement of the GRAPE-6 force engine.
 *
 * TEST INFRASTRUCTURE (the oracle).  Only tests/, the smoke check and the
 * bench's CPU-baseline leg may load this; the engine never calls it.
 *
 * It states, in plain C and FP64 throughout, what the engine behind the
 * g6 ABI (include/grape6.h:16-104) must return, in the spirit of the
 * reference's GRAPE-4 software simulator (src/harpsims/harp3fastsim.c):
 *
 *   predictor   x_p = x + dt (v + dt (a2 + dt j6)),
 *               v_p = v + dt (2 a2 + dt 3 j6),   dt = ti - tj
 *               -- the 3rd-order Taylor step of _dyn_::predict_loworder
 *               (include/_dyn_.h:265-299) written in the a/2, j/6 terms the
 *               adaptor sends (hdyn_grape6.C:230-281);
 *   pair terms  accumulate_acc_and_jerk (hdyn_ev.C:2019-2036):
 *               r2inv = 1/(dr.dr + eps2), a3 = -3 (dr.dv) r2inv,
 *               mrinv = m sqrt(r2inv), pot -= mrinv, a += mrinv r2inv dr,
 *               j += mrinv r2inv (dv + a3 dr);
 *               self excluded by index (hdyn_grape6.C:675 passes index[]);
 *   nn          first j in address order with the smallest dr.dr (no
 *               softening; strict '<' as update_nn_coll, hdyn_inline.C:44);
 *               0 when there is no other particle;
 *   nb lists    {j != self : dr.dr < h2_i} in ascending address, plus i
 *               itself when npipes > 48 and h2_i > 0 (the GPU-engine
 *               convention kira expects, hdyn_grape6.C:2309-2315).
 *
 * Pinned against the reference's own FP64 path (oracle/_ref/libref_force.so
 * over hdyn::flat_calculate_acc_and_jerk) by tests/test_oracle.py and the
 * committed fixtures in tests/golden/.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Predict n j-particles to ti.  Arrays are [n] or [n][3]. */
void g6o_predict(int n, double ti, const double *tj, const double *x,
                 const double *v, const double *a2, const double *j6,
                 double *xp, double *vp)
{
    for (int j = 0; j < n; j++) {
        double dt = ti - tj[j];
        for (int c = 0; c < 3; c++) {
            int k = 3 * j + c;
            xp[k] = x[k] + dt * (v[k] + dt * (a2[k] + dt * j6[k]));
            vp[k] = v[k] + dt * (2.0 * a2[k] + dt * 3.0 * j6[k]);
        }
    }
}

/* Force on ni i-particles from nj predicted j-particles.
 * j: xj/vj [nj][3], mj [nj], jindex [nj]; i: xi/vi [ni][3], index [ni].
 * Outputs acc/jerk [ni][3], pot [ni], nn [ni], nn_r2 [ni] (dr.dr of nn). */
void g6o_force(int nj, const double *xj, const double *vj, const double *mj,
               const int *jindex, int ni, const int *index, const double *xi,
               const double *vi, double eps2, double *acc, double *jerk,
               double *pot, int *nn, double *nn_r2)
{
    for (int i = 0; i < ni; i++) {
        double a[3] = {0, 0, 0}, jk[3] = {0, 0, 0}, p = 0;
        double best = HUGE_VAL;
        int bj = -1;
        const double *x0 = xi + 3 * i, *v0 = vi + 3 * i;
        for (int j = 0; j < nj; j++) {
            if (jindex[j] == index[i]) continue;
            double dr[3], dv[3];
            for (int c = 0; c < 3; c++) {
                dr[c] = xj[3 * j + c] - x0[c];
                dv[c] = vj[3 * j + c] - v0[c];
            }
            double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
            double rv = dr[0] * dv[0] + dr[1] * dv[1] + dr[2] * dv[2];
            double r2inv = 1.0 / (r2 + eps2);
            double a3 = -3.0 * rv * r2inv;
            double mrinv = mj[j] * sqrt(r2inv);
            double mr3inv = mrinv * r2inv;
            p -= mrinv;
            for (int c = 0; c < 3; c++) {
                a[c] += mr3inv * dr[c];
                jk[c] += mr3inv * (dv[c] + a3 * dr[c]);
            }
            if (r2 < best) {
                best = r2;
                bj = j;
            }
        }
        for (int c = 0; c < 3; c++) {
            acc[3 * i + c] = a[c];
            jerk[3 * i + c] = jk[c];
        }
        pot[i] = p;
        nn[i] = bj < 0 ? 0 : bj;
        if (nn_r2) nn_r2[i] = best;
    }
}

/* Neighbour lists.  For each i with h2[i] > 0, writes the ascending
 * addresses into nbl + off[i] and the length into len[i]; off[i+1] =
 * off[i] + len[i] (off has ni+1 entries, caller-sized by a first call with
 * nbl == NULL that only fills len/off).  include_self mirrors npipes > 48. */
void g6o_neighbours(int nj, const double *xj, const int *jindex, int ni,
                    const int *index, const double *xi, const double *h2,
                    int include_self, int *len, long long *off, int *nbl)
{
    long long total = 0;
    for (int i = 0; i < ni; i++) {
        int cnt = 0;
        off[i] = total;
        if (h2[i] > 0) {
            for (int j = 0; j < nj; j++) {
                int hit;
                if (jindex[j] == index[i]) {
                    hit = include_self;
                } else {
                    double r2 = 0;
                    for (int c = 0; c < 3; c++) {
                        double d = xj[3 * j + c] - xi[3 * i + c];
                        r2 += d * d;
                    }
                    hit = r2 < h2[i];
                }
                if (hit) {
                    if (nbl) nbl[total + cnt] = j;
                    cnt++;
                }
            }
        }
        len[i] = cnt;
        total += cnt;
    }
    off[ni] = total;
}
