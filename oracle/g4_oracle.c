/*
 * g4_oracle.c -- FP64 CPU restatement of the GRAPE-4 (HARP-3) pipeline.
 *
 * TEST INFRASTRUCTURE (the oracle).  Only tests/ may load this; the engine
 * never calls it.
 *
 * It restates, in the same operation order, the reference's IEEE GRAPE-4
 * simulator (src/harpsims/harp3fastsim.c), the one executable definition of
 * the GRAPE-4 ABI (include/grape4.h) in the reference tree:
 *
 *   predictor   s = ti - tj;  xp = ((jj s + aj) s + v) s + x;
 *               vp = (jj (1.5 s) + aj) (2 s) + v            (:250-260)
 *               with aj = acc/2, jj = jerk/6 as kira stores them
 *               (hdyn_grape4.C:265-266);
 *   i-side      epsi = 2 eps2[i], hmem = 2 h2[i]             (:240-242);
 *   pair loop   dr2 = epsi + dx dx + dy dy + dz dz, drdv = dr.dv   (:289-299);
 *               neighbour j when dr2 < hmem                  (:300-303);
 *               when dr2 > 0: dr2i = 1/dr2, dr3i = m dr2i sqrt(dr2i),
 *               drdv = 3 drdv dr2i, acc += dr dr3i,
 *               jerk += (dv - dr drdv) dr3i                  (:304-314).
 *
 * The simulator sets pot[i] = 0 and never accumulates it (:281); real
 * GRAPE-4 boards return the potential, which kira's GRAPE-4 energy path
 * reads (hdyn_grape4.C:789-840).  This oracle states it as
 * pot -= m sqrt(dr2i) over the same pairs (the sign of the GRAPE-6
 * convention, pot < 0).
 *
 * Compiled with FP contraction off so that acc, jerk and the neighbour
 * lists reproduce the simulator bit for bit (tests/test_g4_oracle.py checks
 * that against oracle/_ref/libharp3sim.so and the fixtures it generated).
 */
#include <math.h>

void g4o_predict(int n, double ti, const double *tj, const double *x, const double *v, const double *aj,
                 const double *jj, double *xp, double *vp)
{
    for (int j = 0; j < n; j++) {
        double s = ti - tj[j];
        double s1 = 1.5 * s;
        double s2 = 2.0 * s;
        for (int k = 0; k < 3; k++) {
            int q = 3 * j + k;
            xp[q] = ((jj[q] * s + aj[q]) * s + v[q]) * s + x[q];
            vp[q] = (jj[q] * s1 + aj[q]) * s2 + v[q];
        }
    }
}

/* Forces on ni i-slots from nj predicted j.  eps2/h2 are the values the
 * caller passes to h3calc_firsthalf_ (the factor 2 is applied here).
 * nbcount[i] gets the number of neighbours; when nblist is not NULL the
 * first nbcap of them (ascending address) go to nblist[i*nbcap + k]. */
void g4o_force(int nj, const double *xj, const double *vj, const double *mj, int ni, const double *xi,
               const double *vi, const double *eps2, const double *h2, double *acc, double *jerk,
               double *pot, int *nbcount, int *nblist, int nbcap)
{
    for (int i = 0; i < ni; i++) {
        double x0 = xi[3 * i], y0 = xi[3 * i + 1], z0 = xi[3 * i + 2];
        double vx0 = vi[3 * i], vy0 = vi[3 * i + 1], vz0 = vi[3 * i + 2];
        double epsi = 2 * eps2[i];
        double hmem = 2 * h2[i];
        double ax = 0, ay = 0, az = 0, jx = 0, jy = 0, jz = 0, p = 0;
        int nnb = 0;
        for (int j = 0; j < nj; j++) {
            double dx = xj[3 * j] - x0;
            double dy = xj[3 * j + 1] - y0;
            double dz = xj[3 * j + 2] - z0;
            double dvx = vj[3 * j] - vx0;
            double dvy = vj[3 * j + 1] - vy0;
            double dvz = vj[3 * j + 2] - vz0;
            double dr2 = epsi + dx * dx + dy * dy + dz * dz;
            double drdv = dx * dvx + dy * dvy + dz * dvz;
            if (dr2 < hmem) {
                if (nblist && nnb < nbcap) nblist[(long)i * nbcap + nnb] = j;
                nnb++;
            }
            if (dr2 > 0.0) {
                double dr2i = 1.0 / dr2;
                double rinv = sqrt(dr2i);
                double dr3i = mj[j] * dr2i * rinv;
                drdv = 3. * drdv * dr2i;
                ax += dx * dr3i;
                ay += dy * dr3i;
                az += dz * dr3i;
                jx += (dvx - dx * drdv) * dr3i;
                jy += (dvy - dy * drdv) * dr3i;
                jz += (dvz - dz * drdv) * dr3i;
                p -= mj[j] * rinv;
            }
        }
        acc[3 * i] = ax;
        acc[3 * i + 1] = ay;
        acc[3 * i + 2] = az;
        jerk[3 * i] = jx;
        jerk[3 * i + 1] = jy;
        jerk[3 * i + 2] = jz;
        pot[i] = p;
        nbcount[i] = nnb;
    }
}
