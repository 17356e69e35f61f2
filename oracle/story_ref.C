// story_ref.C -- TEST INFRASTRUCTURE (the oracle): the reference's own
// snapshot reader, run on a story-format text.  Linked by
// oracle/build_ref.py against the reference library compiled from its
// sources; nothing here is shipped.
//
// Reads stdin with get_dyn() until it returns NULL, exactly as Starlab's
// tools do (src/node/dyn/util/dyn_io.C:280-296), and prints, per snapshot,
// every node in pre-order with its values as C99 hex floats (exact):
//   P <parent> <index> <name length>:<name> m x y z vx vy vz
// then every leaf's position and velocity relative to the root
// (something_relative_to_root, src/node/dyn/util/dyn_tt.C:94-110):
//   L x y z vx vy vz
// and the static system time after the snapshot:  T t
// With -t it prints nothing but the seconds spent in get_dyn and rmtree
// (the CPU reading time of the reference); with -w it writes every snapshot
// back with the reference's put_node (src/node/util/tree_io.C:412+).
#include "dyn.h"
#include <stdio.h>
#include <string.h>
#include <time.h>

static long long dump(dyn *b, long long parent, long long &next)
{
    const long long me = next++;
    const char *nm = b->get_name();
    vec p = b->get_pos(), v = b->get_vel();
    printf("P %lld %d %d:%s %a %a %a %a %a %a %a\n", parent, b->get_index(), nm ? (int)strlen(nm) : -1,
           nm ? nm : "", (double)b->get_mass(), p[0], p[1], p[2], v[0], v[1], v[2]);
    for_all_daughters(dyn, b, d) dump(d, me, next);
    return me;
}

int main(int argc, char **argv)
{
    const bool timing = argc > 1 && !strcmp(argv[1], "-t");
    const bool write = argc > 1 && !strcmp(argv[1], "-w");
    long long next = 0, roots = 0;
    timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    dyn *b;
    while ((b = get_dyn())) {
        roots++;
        if (write) {
            put_node(b);
        } else if (!timing) {
            dump(b, -1, next);
            for_all_leaves(dyn, b, bi) {
                if (bi == b) continue;  // for_all_leaves includes a root without daughters
                vec p = something_relative_to_root(bi, &dyn::get_pos);
                vec v = something_relative_to_root(bi, &dyn::get_vel);
                printf("L %a %a %a %a %a %a\n", p[0], p[1], p[2], v[0], v[1], v[2]);
            }
            printf("T %a\n", (double)b->get_system_time());
        }
        rmtree(b);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (timing)
        printf("seconds %.6f roots %lld\n", (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec), roots);
    return 0;
}
