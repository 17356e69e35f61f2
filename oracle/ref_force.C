// ref_force.C -- C entry point over the reference's own FP64 force path.
//
// Test infrastructure (oracle), not product.  Builds a flat Starlab tree
// (root + N top-level leaves) from plain arrays, predicts every node to the
// block time with the reference's _dyn_::predict_loworder
// (include/_dyn_.h:265-299), then calls hdyn::flat_calculate_acc_and_jerk
// (src/node/dyn/hdyn/evolve/hdyn_ev.C:2047-2227) for each requested i.  That
// is kira's config-0 (`kira -0`) top-level force path
// (kira_ev.C:877 -> top_level_acc_and_jerk_for_list -> hdyn_ev.C:3755).
//
// Compiled against the reference headers and linked with the reference
// objects by oracle/build_ref.py into oracle/_ref/libref_force.so.

#include "hdyn.h"
#include <vector>
#include <map>
#include <pthread.h>
#include <time.h>

namespace {

struct Shared {
    hdyn *root;
    std::vector<hdyn *> *nodes;
    const int *ilist;
    int ni, nthreads;
};

struct Work {
    Shared *sh;
    int tid;
};

// Round-robin i over threads, each i writing only its own node: the same
// split kira's pthreads driver uses (kira_ev.C:954-1064).
void *force_worker(void *arg)
{
    Work *w = (Work *)arg;
    Shared *sh = w->sh;
    for (int k = w->tid; k < sh->ni; k += sh->nthreads)
        (*sh->nodes)[sh->ilist[k]]->flat_calculate_acc_and_jerk(sh->root, false);
    return NULL;
}

double wall_seconds()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

}  // namespace

extern "C" int ref_flat_force(int n, const double *mass, const double *pos,
                              const double *vel, const double *acc,
                              const double *jerk, const double *tj,
                              double ti, double eps, int ni, const int *ilist,
                              double *acc_out, double *jerk_out,
                              double *pot_out, int *nn_out,
                              double *dnn_sq_out, double *pred_pos_out,
                              double *pred_vel_out, double *eps2_used,
                              int nthreads, double *force_seconds)
// Inputs are per particle (index 0..n-1): mass[n], pos/vel/acc/jerk[n][3],
// tj[n] (time of the last step).  acc and jerk are the full acc and jerk at
// tj (the predictor's old_acc/old_jerk).  eps is the softening length; the
// reference squares it itself (hdyn.h set_eps), and the square it used is
// returned in *eps2_used.  For i = ilist[k] the outputs at k are acc, jerk
// (full jerk), pot, the nearest neighbour's index and its squared distance
// (no softening).  pred_pos_out/pred_vel_out, if non-NULL, receive every
// particle's predicted position and velocity at ti.  nthreads > 1 runs the
// force loop on that many POSIX threads; *force_seconds (if non-NULL)
// receives the wall time of the force loop alone.
{
    if (n <= 0) return -1;
    hdyn *root = new hdyn;
    root->set_root(root);
    std::vector<hdyn *> nodes(n);
    std::map<hdyn *, int> index_of;
    hdyn *prev = NULL;
    for (int i = 0; i < n; i++) {
        hdyn *b = new hdyn;
        nodes[i] = b;
        index_of[b] = i;
        b->set_parent(root);
        if (prev) {
            prev->set_younger_sister(b);
            b->set_elder_sister(prev);
        } else {
            root->set_oldest_daughter(b);
        }
        prev = b;
    }
    real mtot = 0;
    for (int i = 0; i < n; i++) {
        hdyn *b = nodes[i];
        b->set_root(root);
        b->set_mass(mass[i]);
        mtot += mass[i];
        b->set_pos(vec(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]));
        b->set_vel(vec(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]));
        vec a(acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]);
        vec j(jerk[3 * i], jerk[3 * i + 1], jerk[3 * i + 2]);
        b->set_acc(a);
        b->set_jerk(j);
        b->set_old_acc(a);
        b->set_old_jerk(j);
        b->set_time(tj[i]);
        b->set_timestep(1);
    }
    root->set_mass(mtot);
    root->set_eps(eps);
    if (eps2_used) *eps2_used = root->get_eps2();
    root->set_system_time(ti);

    // Prediction of every top-level node to the block time, as kira does
    // before the CPU force loop (kira.C:1234).
    predict_loworder_all(root, ti);

    if (pred_pos_out || pred_vel_out) {
        for (int i = 0; i < n; i++) {
            vec p = nodes[i]->get_pred_pos();
            vec v = nodes[i]->get_pred_vel();
            for (int k = 0; k < 3; k++) {
                if (pred_pos_out) pred_pos_out[3 * i + k] = p[k];
                if (pred_vel_out) pred_vel_out[3 * i + k] = v[k];
            }
        }
    }

    for (int k = 0; k < ni; k++)
        if (ilist[k] < 0 || ilist[k] >= n) return -2;
    if (nthreads < 1) nthreads = 1;
    double t0 = wall_seconds();
    if (nthreads == 1) {
        for (int k = 0; k < ni; k++)
            nodes[ilist[k]]->flat_calculate_acc_and_jerk(root, false);
    } else {
        Shared sh;
        sh.root = root; sh.nodes = &nodes; sh.ilist = ilist;
        sh.ni = ni; sh.nthreads = nthreads;
        std::vector<Work> work(nthreads);
        std::vector<pthread_t> th(nthreads);
        for (int t = 0; t < nthreads; t++) {
            work[t].sh = &sh;
            work[t].tid = t;
            pthread_create(&th[t], NULL, force_worker, &work[t]);
        }
        for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    }
    if (force_seconds) *force_seconds = wall_seconds() - t0;

    for (int k = 0; k < ni; k++) {
        hdyn *b = nodes[ilist[k]];
        vec a = b->get_acc(), j = b->get_jerk();
        for (int c = 0; c < 3; c++) {
            acc_out[3 * k + c] = a[c];
            jerk_out[3 * k + c] = j[c];
        }
        pot_out[k] = b->get_pot();
        hdyn *nn = b->get_nn();
        nn_out[k] = nn ? index_of[nn] : -1;
        dnn_sq_out[k] = b->get_d_nn_sq();
    }

    // Tear down without running the reference's recursive destructors over
    // a 10^5-node sibling chain.
    for (int i = 0; i < n; i++) {
        nodes[i]->set_parent(NULL);
        nodes[i]->set_elder_sister(NULL);
        nodes[i]->set_younger_sister(NULL);
        delete nodes[i];
    }
    root->set_oldest_daughter(NULL);
    delete root;
    return 0;
}
