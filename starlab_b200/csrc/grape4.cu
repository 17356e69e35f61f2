// grape4.cu -- the extern "C" h3* entry points of libh3b200.so: Starlab's
// GRAPE-4 (HARP-3) host-library ABI (include/grape4.h:22-45) over one Engine
// instance running the GRAPE-4 pipeline variant of the FP64 force kernel.
//
// The caller is kira's GRAPE-4 branch (src/node/dyn/hdyn/evolve/
// hdyn_grape4.C), single-threaded with global state, like the simulator it
// replaces (src/harpsims/harp3fastsim.c), so this layer keeps one global
// state too.  What it adds over a plain forward to the engine:
//   * DMA buffers: h3mjpdma_indirect_ gathers host elements hostindex[i]-1
//     into buffer buff_id; h3mjpdma_start_ commits a buffer to j-memory
//     (harp3fastsim.c:140-206);
//   * the simulator's factor 2 on eps2 and h2 (harp3fastsim.c:240-242);
//   * i-slot deduplication: kira pads every call to h3npipe_() slots with
//     copies of its last i and, built with USE_HALF_CHIP, gives each i two
//     slots (hdyn_grape4.C:350-382); runs of consecutive bit-identical slots
//     are computed once and their results copied, which is exact because a
//     slot's results depend only on its own inputs;
//   * neighbour lists of any length (h3nblist_ has no length argument).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "engine.h"
// The library is built with hidden visibility; only the C ABI is exported.
#pragma GCC visibility push(default)
#include "../../include/h3b200.h"
#pragma GCC visibility pop

namespace {

constexpr int kBuffers = 64;
constexpr int kJpMax = 1 << 20;

struct JEntry {
    int addr;
    double x[3], v[3], a2[3], j6[3], m, t;
};

struct State {
    g6::Engine *eng = nullptr;
    double ti = 0;
    std::vector<JEntry> buf[kBuffers];
    int buff_used = 0;
    // last call: slots -> distinct records
    int ni = 0, nu = 0;
    std::vector<int> slot;
    std::vector<double> xu, vu, eu, hu;
    std::vector<double> acc, jerk, pot;
    bool pending = false, have_results = false, nb_read = false;
    long long calls = 0, slots = 0, computed = 0, interactions = 0, j_updates = 0;
};

State g;
std::string g_err;

int env_int(const char *name, int dflt) {
    const char *s = getenv(name);
    return (s && *s) ? atoi(s) : dflt;
}

int npipes() {
    static const int n = [] {
        int v = env_int("H3B200_NPIPES", 4096);
        return v < 1 ? 1 : v;
    }();
    return n;
}

[[noreturn]] void die(const std::string &msg) {
    g_err = msg;
    fprintf(stderr, "%s\n", msg.c_str());
    fflush(stderr);
    exit(-1);
}

g6::Engine &engine() {
    if (!g.eng) g.eng = new g6::Engine(0);
    if (!g.eng->is_open()) {
        if (g.eng->open(env_int("G6B200_DEVICE", 0), 0)) die("h3b200: open failed: " + g.eng->last_error);
        g.eng->set_mode(g6::kModeF64);
        g.eng->set_npipes(npipes());
    }
    return *g.eng;
}

void check_buffer(int b, const char *who) {
    if (b < 0 || b >= kBuffers) {
        char m[128];
        snprintf(m, sizeof m, "(%s) DMA buffer id %d outside [0, %d)", who, b, kBuffers);
        die(m);
    }
}

void commit(int b) {
    g6::Engine &e = engine();
    for (const JEntry &q : g.buf[b]) {
        if (e.set_j(q.addr, q.addr, q.t, q.m, nullptr, q.j6, q.a2, q.v, q.x))
            die("(h3mjpdma_start) " + e.last_error);
        g.j_updates++;
    }
}

// Collect the results of the pending call into the per-record arrays.
void finish() {
    if (!g.pending) return;
    g.pending = false;
    g.acc.resize(3 * (size_t)g.nu);
    g.jerk.resize(3 * (size_t)g.nu);
    g.pot.resize(g.nu);
    g6::Engine &e = engine();
    int rc = e.lasthalf(g.nu, reinterpret_cast<double(*)[3]>(g.acc.data()),
                        reinterpret_cast<double(*)[3]>(g.jerk.data()), g.pot.data(), nullptr);
    if (rc) die("(h3calc_lasthalf) engine error: " + e.last_error);
    g.have_results = true;
    g.nb_read = false;
}

bool same_slot(const double (*xi)[3], const double (*vi)[3], const double *eps2, const double *h2, int a, int b) {
    return !memcmp(xi[a], xi[b], sizeof(double) * 3) && !memcmp(vi[a], vi[b], sizeof(double) * 3) &&
           !memcmp(&eps2[a], &eps2[b], sizeof(double)) && !memcmp(&h2[a], &h2[b], sizeof(double));
}

int record_of(int chip) {
    if (!g.have_results || chip < 0 || chip >= g.ni) return -1;
    return g.slot[chip];
}

void read_lists() {
    finish();
    if (!g.have_results) die("(h3nbread) no force call to read neighbour lists from");
    if (g.nb_read) return;
    g6::Engine &e = engine();
    // 1 = some list is longer than the force pass keeps per i; those pipes
    // are recomputed in full by neighbours_all.
    if (e.read_neighbours() < 0) die("(h3nbread) " + e.last_error);
    g.nb_read = true;
}

}  // namespace

extern "C" {

void h3open_(void) { engine(); }

void h3close_(void) {
    if (g.eng) g.eng->close();
    for (auto &b : g.buf) b.clear();
    g.buff_used = 0;
    g.pending = g.have_results = g.nb_read = false;
    g.ni = g.nu = 0;
}

int h3npipe_(void) { return npipes(); }

void h3setnboards_(int *) {}

int h3getnboards_(void) { return 1; }

unsigned int h3wait_(void) { return 0; }

void h3setti_(double *ti) { g.ti = *ti; }

void h3setmode_(int *, int *) {}

void h3setled_(int *, int *) {}

int h3jpmax_(void) { return kJpMax; }

void h3mjpdma_indirect_(int *nj, int *hostindex, double xj[][3], double vj[][3], double aj[][3], double jj[][3],
                        double *mj, double *tj, int *, int *buff_id) {
    const int n = *nj;
    if (n > kJpMax || n < 0) {
        char m[128];
        snprintf(m, sizeof m, "(h3jpdma) Too large nj (%d > %d)", n, kJpMax);
        die(m);
    }
    const int b = (buff_id && *buff_id >= 0) ? *buff_id : g.buff_used++;
    check_buffer(b, "h3mjpdma_indirect");
    std::vector<JEntry> &B = g.buf[b];
    B.resize(n);
    for (int i = 0; i < n; ++i) {
        const int h = hostindex[i] - 1;
        if (h < 0) die("(h3mjpdma_indirect) host index below 1");
        JEntry &q = B[i];
        q.addr = h;
        for (int c = 0; c < 3; ++c) {
            q.x[c] = xj[h][c];
            q.v[c] = vj[h][c];
            q.a2[c] = aj[h][c];
            q.j6[c] = jj[h][c];
        }
        q.m = mj[h];
        q.t = tj[h];
    }
}

void h3jpdma_indirect_(int *nj, int *hostindex, double xj[][3], double vj[][3], double aj[][3], double jj[][3],
                       double *mj, double *tj, int *mode) {
    int zero = 0;
    h3mjpdma_indirect_(nj, hostindex, xj, vj, aj, jj, mj, tj, mode, &zero);
    h3mjpdma_start_(&zero);
}

void h3mjpdma_start_(int *buff_id) {
    check_buffer(*buff_id, "h3mjpdma_start");
    commit(*buff_id);
}

void h3mjpdma_flush_(void) {
    for (int b = 0; b < g.buff_used && b < kBuffers; ++b) commit(b);
    g.buff_used = 0;
}

void h3jpdma_flush_(void) { h3mjpdma_flush_(); }

void h3jpdma_reset_(void) { g.buff_used = 0; }

void h3calc_firsthalf_(int *nj, int *ni, double xi[][3], double vi[][3], double *eps2, double *h2) {
    const int n = *ni, m = *nj;
    if (n > npipes() || n < 0) {
        char msg[128];
        snprintf(msg, sizeof msg, "(h3ipdma) Too large ni (%d > %d)", n, npipes());
        die(msg);
    }
    g6::Engine &e = engine();
    finish();  // a call whose results were never read
    g.slot.resize(n);
    g.xu.clear();
    g.vu.clear();
    g.eu.clear();
    g.hu.clear();
    int nu = 0;
    for (int k = 0; k < n; ++k) {
        if (k > 0 && same_slot(xi, vi, eps2, h2, k, k - 1)) {
            g.slot[k] = g.slot[k - 1];
            continue;
        }
        g.slot[k] = nu++;
        g.xu.insert(g.xu.end(), xi[k], xi[k] + 3);
        g.vu.insert(g.vu.end(), vi[k], vi[k] + 3);
        g.eu.push_back(2.0 * eps2[k]);
        g.hu.push_back(2.0 * h2[k]);
    }
    e.set_ti(g.ti);
    if (e.firsthalf_g4(m, nu, reinterpret_cast<const double(*)[3]>(g.xu.data()),
                       reinterpret_cast<const double(*)[3]>(g.vu.data()), g.eu.data(), g.hu.data()))
        die("(h3calc_firsthalf) " + e.last_error);
    g.ni = n;
    g.nu = nu;
    g.pending = true;
    g.have_results = false;
    g.nb_read = false;
    g.calls++;
    g.slots += n;
    g.computed += nu;
    g.interactions += (long long)nu * m;
}

void h3calc_lasthalf_(int *ni, double acc[][3], double jerk[][3], double *pot) {
    finish();
    if (!g.have_results) die("(h3calc_lasthalf) no h3calc_firsthalf_ call to complete");
    const int n = *ni;
    if (n > g.ni || n < 0) {
        char msg[128];
        snprintf(msg, sizeof msg, "(h3calc_lasthalf) ni %d above the %d slots of the call", n, g.ni);
        die(msg);
    }
    for (int k = 0; k < n; ++k) {
        const int u = g.slot[k];
        for (int c = 0; c < 3; ++c) {
            acc[k][c] = g.acc[3 * (size_t)u + c];
            jerk[k][c] = g.jerk[3 * (size_t)u + c];
        }
        pot[k] = g.pot[u];
    }
}

void h3calc_(int *nj, int *ni, double xi[][3], double vi[][3], double *eps2, double *h2, double acc[][3],
             double jerk[][3], double *pot) {
    h3calc_firsthalf_(nj, ni, xi, vi, eps2, h2);
    h3calc_lasthalf_(ni, acc, jerk, pot);
}

void h3nbread_(int *) { read_lists(); }

int h3nblist_(int *, int *chip, int *nblist) {
    read_lists();
    const int u = record_of(*chip);
    if (u < 0) return 0;
    const int n = engine().neighbours_all(u, nblist);
    if (n < 0) die("(h3nblist) " + engine().last_error);
    return n;
}

int count_nblist_low(int, int chip) {
    read_lists();
    const int u = record_of(chip);
    if (u < 0) return 0;
    const int n = engine().neighbour_count(u);
    return n < 0 ? 0 : n;
}

void h3setdebuglevel_(int *) {}

void h3checkdmabuffers_(void) {}

void set_time_check_mode(int) {}

const char *h3b200_last_error(void) { return g_err.c_str(); }

int h3b200_get_stats(h3b200_stats *out) {
    if (!out) return -1;
    out->calls = g.calls;
    out->slots = g.slots;
    out->computed = g.computed;
    out->interactions = g.interactions;
    out->j_updates = g.j_updates;
    out->launches = g.eng ? g.eng->stats().launches : 0;
    return 0;
}

}  // extern "C"
