/* Stand-in for Starlab's Fortran-77 triple-stability test (reference file
 * src/node/dyn/hdyn/evolve/nstab.f, called from mardling_unstable.C:52).
 * No Fortran compiler exists in this image, so the oracle build links this
 * instead.  It answers "unstable" (1), the conservative choice: kira then
 * never treats a hierarchical triple as a stable multiple.  The force-path
 * oracle runs (Plummer spheres without primordial binaries, at most one
 * N-body time unit) never reach it; a counter records whether they did.
 * Test infrastructure only. */
#include <stdio.h>

int nstab_calls_oracle_stub = 0;

int nstab_(double *sigma, double *ei0, double *eo, double *relinc,
           double *m1, double *m2, double *m3)
{
    (void)sigma; (void)ei0; (void)eo; (void)relinc; (void)m1; (void)m2; (void)m3;
    if (nstab_calls_oracle_stub++ == 0)
        fprintf(stderr, "oracle nstab stub: answering 'unstable'\n");
    return 1;
}
