// abi.cu -- the extern "C" g6_* entry points of libg6b200.so.
//
// Each maps one call of Starlab's GRAPE-6 ABI (include/grape6.h:16-104) onto
// an Engine instance keyed by cluster_id.  The caller is single-threaded
// (hdyn_grape6.C keeps global state, :86-124); a mutex still guards the
// instance table so that independent host threads may drive different
// cluster ids.
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include "engine.h"
// The library is built with hidden visibility; only the C ABI is exported.
#pragma GCC visibility push(default)
#include "../../include/g6b200.h"
#pragma GCC visibility pop

namespace {

std::mutex g_mu;
std::map<int, std::unique_ptr<g6::Engine>> g_engines;
int g_open_device = -1;
int g_open_nmax = 0;
thread_local std::string g_err;

int default_device() {
    if (g_open_device >= 0) return g_open_device;
    const char *s = getenv("G6B200_DEVICE");
    return (s && *s) ? atoi(s) : 0;
}

g6::Engine *engine(int id, bool open = true) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_engines.find(id);
    g6::Engine *e;
    if (it == g_engines.end()) {
        e = new g6::Engine(id);
        g_engines[id].reset(e);
    } else {
        e = it->second.get();
    }
    if (open && !e->is_open()) {
        if (e->open(default_device(), g_open_nmax)) {
            g_err = e->last_error;
            return nullptr;
        }
    }
    return e;
}

int cid(const int *p) { return p ? *p : 0; }

void note(g6::Engine *e) {
    if (e && !e->last_error.empty()) g_err = e->last_error;
}

}  // namespace

namespace g6 {
// Lets other translation units of the library set g6b200_last_error().
void record_error(const std::string &msg) { g_err = msg; }
}  // namespace g6

extern "C" {

void g6_set_tunit_(int *) {}
void g6_set_xunit_(int *) {}

int g6_open_(int *cluster_id) {
    g6::Engine *e = engine(cid(cluster_id));
    return e ? 0 : -1;
}

int g6_close_(int *cluster_id) {
    g6::Engine *e = engine(cid(cluster_id), false);
    e->close();
    return 0;
}

int g6_open_special2(int ngpu, int *list, int nmax) {
    if (ngpu > 0 && list) g_open_device = list[0];
    if (nmax > 0) g_open_nmax = nmax;
    int zero = 0;
    return g6_open_(&zero);
}

int g6_open_special(int ngpu, int *list) { return g6_open_special2(ngpu, list, 0); }

int g6_reset_(int *cluster_id) {
    g6::Engine *e = engine(cid(cluster_id), false);
    return e->reset();
}

int g6_reset_fofpga_(int *cluster_id) { return g6_reset_(cluster_id); }

int g6_npipes_(void) {
    // Reported without opening the device: kira asks during configuration.
    g6::Engine *e = engine(0, false);
    return e->npipes();
}

void g6_set_ti_(int *cluster_id, double *ti) {
    g6::Engine *e = engine(cid(cluster_id));
    if (e && ti) e->set_ti(*ti);
}

int g6_set_j_particle_(int *cluster_id, int *address, int *index, double *tj, double *dtj, double *mass,
                       double k18[3], double j6[3], double a2[3], double v[3], double x[3]) {
    (void)dtj;
    g6::Engine *e = engine(cid(cluster_id));
    if (!e) return -1;
    int rc = e->set_j(*address, index ? *index : *address, *tj, *mass, k18, j6, a2, v, x);
    if (rc) note(e);
    return rc;
}

void g6calc_firsthalf_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3], double vi[][3],
                       double aold[][3], double j6old[][3], double phiold[], double *eps2, double h2[]) {
    (void)aold;
    (void)j6old;
    (void)phiold;
    g6::Engine *e = engine(cid(cluster_id));
    if (!e) return;
    if (e->firsthalf(*nj, *ni, index, xi, vi, eps2 ? *eps2 : 0.0, h2)) note(e);
}

int g6calc_lasthalf_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3], double vi[][3],
                     double *eps2, double h2[], double acc[][3], double jerk[][3], double pot[]) {
    (void)nj; (void)index; (void)xi; (void)vi; (void)eps2; (void)h2;
    g6::Engine *e = engine(cid(cluster_id));
    if (!e) return -1;
    int rc = e->lasthalf(*ni, acc, jerk, pot, nullptr);
    if (rc) note(e);
    return rc;
}

int g6calc_lasthalf2_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3], double vi[][3],
                      double *eps2, double h2[], double acc[][3], double jerk[][3], double pot[],
                      int nnbindex[]) {
    (void)nj; (void)index; (void)xi; (void)vi; (void)eps2; (void)h2;
    g6::Engine *e = engine(cid(cluster_id));
    if (!e) return -1;
    int rc = e->lasthalf(*ni, acc, jerk, pot, nnbindex);
    if (rc) note(e);
    return rc;
}

int g6_read_neighbour_list_(int *cluster_id) {
    g6::Engine *e = engine(cid(cluster_id));
    if (!e) return -1;
    int rc = e->read_neighbours();
    if (rc < 0) note(e);
    return rc;
}

int g6_read_neighbour_list_old_(int *cluster_id) { return g6_read_neighbour_list_(cluster_id); }

int g6_get_neighbour_list_(int *cluster_id, int *pipe, int *max_length, int *nblen, int nbl[]) {
    g6::Engine *e = engine(cid(cluster_id));
    if (!e) return -1;
    return e->get_neighbours(*pipe, *max_length, nblen, nbl);
}

int g6_initialize_jp_buffer_(int *clusterid, int *size) {
    (void)size;
    return engine(cid(clusterid)) ? 0 : -1;
}

int g6_flush_jp_buffer_(int *clusterid) {
    g6::Engine *e = engine(cid(clusterid));
    if (!e) return -1;
    int rc = e->flush_j();
    if (rc) note(e);
    return rc;
}

void g6_set_neighbour_list_sphere_(int *cluster_id, double *h2) {
    g6::Engine *e = engine(cid(cluster_id), false);
    if (h2) e->set_default_h2(*h2);
}

int g6b200_set_precision(int cluster_id, int mode) {
    g6::Engine *e = engine(cluster_id, false);
    return e->set_mode(mode);
}

int g6b200_get_precision(int cluster_id) { return engine(cluster_id, false)->mode(); }

int g6b200_set_npipes(int cluster_id, int npipes) { return engine(cluster_id, false)->set_npipes(npipes); }

int g6b200_get_npipes(int cluster_id) { return engine(cluster_id, false)->npipes(); }

int g6b200_set_config(int cluster_id, int il, int r, int warps, int h, int nsplit) {
    g6::ForceConfig c{};
    c.il = il;
    c.r = r;
    c.warps = warps;
    c.H = h;
    c.nsplit = nsplit;
    if (il != 0) {
        bool ok = (il == 1 || il == 8 || il == 32) && (r == 1 || ((r == 2 || r == 4) && il == 32)) && warps >= 1 &&
                  warps <= 8 && (warps & (warps - 1)) == 0 && h >= 1 && warps % h == 0 && nsplit >= 1;
        if (!ok) {
            g_err = "g6b200_set_config: unsupported configuration";
            return -1;
        }
    }
    engine(cluster_id, false)->set_config_override(c);
    return 0;
}

int g6b200_get_config(int cluster_id, int *out5) {
    const g6::ForceConfig &c = engine(cluster_id, false)->last_config();
    out5[0] = c.il;
    out5[1] = c.r;
    out5[2] = c.warps;
    out5[3] = c.H;
    out5[4] = c.nsplit;
    return 0;
}

int g6b200_set_j_particles(int cluster_id, int n, const int *address, const int *index, const double *tj,
                           const double *mass, const double (*k18)[3], const double (*j6)[3],
                           const double (*a2)[3], const double (*v)[3], const double (*x)[3]) {
    g6::Engine *e = engine(cluster_id);
    if (!e) return -1;
    if (e->set_j_bulk(n, address, index, tj, mass, k18 ? &k18[0][0] : nullptr, &j6[0][0], &a2[0][0], &v[0][0],
                      &x[0][0])) {
        note(e);
        return -1;
    }
    return 0;
}

int g6b200_sweep(int cluster_id, int nj, int i0, int ni, double eps2, double (*acc)[3], double (*jerk)[3],
                 double *pot, int *nn) {
    g6::Engine *e = engine(cluster_id);
    if (!e) return -1;
    const bool copy = acc || jerk || pot || nn;
    int rc = e->sweep(nj, i0, ni, eps2, copy, acc, jerk, pot, nn);
    if (rc) note(e);
    return rc;
}

int g6b200_calc_pot(int cluster_id, int nj, int ni, const int *index, const double (*xi)[3], double eps2,
                    double *pot) {
    g6::Engine *e = engine(cluster_id);
    if (!e) return -1;
    int rc = e->potential(nj, ni, index, xi, eps2, pot);
    if (rc) note(e);
    return rc;
}

int g6b200_energies(int cluster_id, int nj, double eps2, double *epot, double *ekin, double *pot) {
    g6::Engine *e = engine(cluster_id);
    if (!e) return -1;
    int rc = e->energies(nj, eps2, epot, ekin, pot);
    if (rc) note(e);
    return rc;
}

int g6b200_split_begin(int cluster_id, int nj, int ni, const int *index, const double (*xi)[3],
                       const double (*vi)[3], double eps2, int block_j, long long *agree, void *stream) {
    g6::Engine *e = engine(cluster_id);
    if (!e) return -1;
    int rc = e->split_begin(nj, ni, index, xi, vi, eps2, block_j, agree, stream);
    if (rc) note(e);
    return rc;
}

int g6b200_split_fix(int cluster_id, long long nblocks_total, long long j_offset, const long long *agree,
                     long long *sums, long long *negj, void *stream) {
    g6::Engine *e = engine(cluster_id);
    if (!e) return -1;
    int rc = e->split_fix(nblocks_total, j_offset, agree, sums, negj, stream);
    if (rc) note(e);
    return rc;
}

int g6b200_split_finish(int cluster_id, long long nblocks_total, long long nj_total, const long long *agree,
                        const long long *sums, const long long *negj, void *stream, double (*acc)[3],
                        double (*jerk)[3], double *pot, int *nn) {
    g6::Engine *e = engine(cluster_id);
    if (!e) return -1;
    int rc = e->split_finish(nblocks_total, nj_total, agree, sums, negj, stream, acc, jerk, pot, nn);
    if (rc) note(e);
    return rc;
}

int g6b200_set_position_range(int cluster_id, double xmax) {
    g6::Engine *e = engine(cluster_id, false);
    e->set_position_range(xmax);
    return 0;
}

int g6b200_get_stats(int cluster_id, g6b200_stats *out) {
    const g6::EngineStats &s = engine(cluster_id, false)->stats();
    out->calls = s.calls;
    out->interactions = s.interactions;
    out->j_updates = s.j_updates;
    out->h2d_bytes = s.h2d_bytes;
    out->d2h_bytes = s.d2h_bytes;
    out->last_force_ms = s.last_force_ms;
    out->last_predict_ms = s.last_predict_ms;
    out->last_call_ms = s.last_call_ms;
    out->launches = s.launches;
    out->refined = s.refined;
    return 0;
}

int g6b200_selftest_copy_timeout(int cluster_id, double limit_ms) {
    g6::Engine *e = engine(cluster_id);
    if (!e) return -1;
    const int rc = e->selftest_copy_timeout(limit_ms);
    if (rc) note(e);
    return rc;
}

const char *g6b200_last_error(void) { return g_err.c_str(); }

}  // extern "C"
