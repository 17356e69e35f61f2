// engine.cu -- host side of one GRAPE-6 engine instance.
//
// Call pipeline (one CUDA stream per instance, everything asynchronous
// until lasthalf):
//   set_j            host staging, deduplicated per address (last write
//                    wins), pinned memory
//   firsthalf        staged j -> device (one copy + scatter kernel);
//                    predictor, only when the block time, nj, the j-state or
//                    the fixed-point range changed (kira calls firsthalf once
//                    per npipes-chunk of a block at the same time);
//                    i-records -> device; force kernel (+ split reduction);
//                    neighbour-list compaction when any h2 > 0;
//                    results -> pinned host memory
//   lasthalf         wait, check the device status word, copy out.
// This is the host-side counterpart of the GRAPE-6 library that
// hdyn_grape6.C drives (send_j_node_to_grape :273, force_by_grape :474-910).
#include "engine.h"
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>

namespace g6 {

namespace {

// Host-side work of large uploads and i-blocks split over up to 8 threads
// (single-threaded memory copies run at a fraction of the host's bandwidth).
// f(lo, hi, t) handles [lo, hi) as thread t; returns when all are done.
// Threads are started per use, so callers ask for one only per
// min_per_thread items (tens of thousands): starting one costs tens of us.
template <class F>
void parallel_ranges(size_t n, size_t min_per_thread, F &&f) {
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>(std::min<size_t>(hw, 8), std::max<size_t>(1, n / min_per_thread));
    if (nt <= 1) {
        f(size_t(0), n, size_t(0));
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    for (size_t t = 1; t < nt; ++t) th.emplace_back([&, t] { f(n * t / nt, n * (t + 1) / nt, t); });
    f(size_t(0), n / nt, size_t(0));
    for (auto &x : th) x.join();
}

int env_int(const char *name, int dflt) {
    const char *s = getenv(name);
    if (!s || !*s) return dflt;
    return atoi(s);
}

long long env_ll(const char *name, long long dflt) {
    const char *s = getenv(name);
    if (!s || !*s) return dflt;
    return atoll(s);
}

int round_up(int x, int m) { return (x + m - 1) / m * m; }

constexpr int kRecMax = 64;  // largest j-record (JRecF64)
constexpr int kPadTile = 256;

// Output buffer layout for a call with ni i-particles.
struct OutLayout {
    size_t status, acc, jerk, pot, nn, total;
    explicit OutLayout(int ni) {
        status = 0;
        acc = 16;
        jerk = acc + 24 * (size_t)ni;
        pot = jerk + 24 * (size_t)ni;
        nn = pot + 8 * (size_t)ni;
        total = nn + 4 * (size_t)ni;
    }
};

}  // namespace

Engine::Engine(int cluster_id) : cluster_id_(cluster_id) {
    npipes_ = env_int("G6B200_NPIPES", 256);
    if (npipes_ < 1) npipes_ = 1;
    nb_cap_ = std::min(std::max(env_int("G6B200_NBMAX", 4096), 16), 8192);
    const char *pm = getenv("G6B200_PRECISION");
    if (pm && (!strcmp(pm, "mixed") || !strcmp(pm, "1"))) mode_ = kModeMixed;
    const char *ml = getenv("G6B200_MIXED_LAYOUT");
    if (ml && !strcmp(ml, "scalar")) mixed_layout_ = kKernMixedDS;
    fault_lasthalf_at_ = env_ll("G6B200_FAULT_LASTHALF", -1);
    event_timing_ = getenv("G6B200_EVENT_TIMING") != nullptr;
    fault_pot_at_ = env_ll("G6B200_FAULT_POT", -1);
    small_enabled_ = env_int("G6B200_SMALL_CALLS", 1) != 0;
    refine_enabled_ = env_int("G6B200_REFINE", 1) != 0;
    mixed_min_work_ = env_ll("G6B200_MIXED_MIN_WORK", 1LL << 25);
}

Engine::~Engine() { close(); }

int Engine::fail(const char *what, cudaError_t e) {
    char buf[256];
    snprintf(buf, sizeof buf, "g6b200[%d]: %s: %s", cluster_id_, what,
             e == cudaSuccess ? "error" : cudaGetErrorString(e));
    last_error = buf;
    return -1;
}

#define G6_CHECK(call, what)                      \
    do {                                          \
        cudaError_t e_ = (call);                  \
        if (e_ != cudaSuccess) return fail(what, e_); \
    } while (0)

int Engine::open(int device, int nmax_hint) {
    if (open_) return 0;
    device_ = device;
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    G6_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    G6_CHECK(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, device_), "attr");
    cudaEvent_t *evs[] = {&ev_stage_, &ev_begin_, &ev_pred0_, &ev_pred1_, &ev_force0_, &ev_force1_, &ev_done_};
    for (cudaEvent_t *e : evs) G6_CHECK(cudaEventCreate(e), "event");
    G6_CHECK(cudaEventCreateWithFlags(&ev_ext_, cudaEventDisableTiming), "event");
    stage_cap_ = 16384;
    G6_CHECK(cudaMallocHost(&h_stage_vals_, sizeof(double) * JF_COUNT * stage_cap_), "pinned stage");
    G6_CHECK(cudaMallocHost(&h_stage_addr_, sizeof(int) * stage_cap_), "pinned stage");
    G6_CHECK(cudaMallocHost(&h_stage_index_, sizeof(int) * stage_cap_), "pinned stage");
    G6_CHECK(cudaMalloc(&d_stage_vals_, sizeof(double) * JF_COUNT * stage_cap_), "stage");
    G6_CHECK(cudaMalloc(&d_stage_addr_, sizeof(int) * stage_cap_), "stage");
    G6_CHECK(cudaMalloc(&d_stage_index_, sizeof(int) * stage_cap_), "stage");
    G6_CHECK(cudaMalloc(&d_energy_, sizeof(double) * (2 * kEnergyBlocks + 2)), "energy");
    G6_CHECK(cudaMallocHost(&h_energy_, sizeof(double) * 2), "energy");
    G6_CHECK(cudaMallocHost(&h_ref_count_, sizeof(int)), "refine");
    *h_ref_count_ = 0;
    G6_CHECK(cudaMalloc(&d_v2_, sizeof(double) * (kRefineBlocks + 1)), "refine");
    G6_CHECK(cudaMalloc(&d_ref_small_, sizeof(int) * 8), "refine");
    G6_CHECK(cudaMemset(d_ref_small_, 0, sizeof(int) * 8), "refine");  // flag count and block counter start at 0
    G6_CHECK(cudaMalloc(&d_ref_items_, sizeof(ForceParams)), "refine");
    open_ = true;
    if (ensure_capacity(std::max(nmax_hint, 1024) - 1)) return -1;
    return 0;
}

void Engine::close() {
    if (!open_) return;
    if (getenv("G6B200_TRACE")) {
        fprintf(stderr,
                "g6b200[%d] trace: calls %lld interactions %lld launches %lld predictions %lld nb_calls %lld "
                "pair_calls %lld refined %lld range_retries %lld grows %lld wait_ms %.1f host_ms %.1f mode %d\n",
                cluster_id_, stats_.calls, stats_.interactions, stats_.launches, stats_.predictions, stats_.nb_calls,
                stats_.pair_calls, stats_.refined, stats_.range_retries, stats_.grows, stats_.wait_ms, stats_.host_ms,
                mode_);
    }
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    auto dfree = [](void *p) { if (p) cudaFree(p); };
    auto hfree = [](void *p) { if (p) cudaFreeHost(p); };
    dfree(d_jraw_); dfree(d_jindex_); dfree(d_jrec_);
    dfree(d_stage_vals_); dfree(d_stage_addr_); dfree(d_stage_index_);
    dfree(d_irec_); dfree(d_out_); dfree(d_part_); dfree(d_tile_cnt_);
    dfree(d_nb_count_); dfree(d_nb_list_); dfree(d_nb_sorted_); dfree(d_nb_off_); dfree(d_bulk_);
    hfree(h_stage_vals_); hfree(h_stage_addr_); hfree(h_stage_index_);
    hfree(h_irec_); hfree(h_out_); hfree(h_nb_off_); hfree(h_nb_count_); hfree(h_bulk_);
    hfree(h_ieps2_); dfree(d_ieps2_); hfree(h_energy_); dfree(d_energy_);
    hfree(h_ref_count_); dfree(d_v2_); dfree(d_ref_small_); dfree(d_ref_items_); dfree(d_q_);
    dfree(d_ref_list_); dfree(d_ref_tcnt_); dfree(d_ref_irec_);
    dfree(d_ref_part_); dfree(d_jrec64_);
    h_ref_count_ = nullptr; d_v2_ = nullptr; d_ref_small_ = nullptr; d_ref_items_ = nullptr; d_q_ = nullptr;
    d_ref_list_ = nullptr; d_ref_tcnt_ = nullptr; d_ref_irec_ = nullptr;
    d_ref_part_ = nullptr; d_jrec64_ = nullptr; ref_cap_ = 0; jrec64_cap_ = 0;
    pred64_valid_ = v2_valid_ = false;
    cudaEvent_t evs[] = {ev_stage_, ev_begin_, ev_pred0_, ev_pred1_, ev_force0_, ev_force1_, ev_done_};
    for (cudaEvent_t e : evs) if (e) cudaEventDestroy(e);
    if (ev_ext_) cudaEventDestroy(ev_ext_);
    ev_ext_ = nullptr;
    cudaStreamDestroy(stream_);
    d_jraw_ = nullptr; d_jindex_ = nullptr; d_jrec_ = nullptr;
    d_stage_vals_ = nullptr; d_stage_addr_ = nullptr; d_stage_index_ = nullptr;
    d_irec_ = nullptr; d_out_ = nullptr; d_part_ = nullptr; d_tile_cnt_ = nullptr;
    d_nb_count_ = nullptr; d_nb_list_ = nullptr; d_nb_sorted_ = nullptr; d_nb_off_ = nullptr;
    d_bulk_ = nullptr; bulk_cap_ = 0; bulk_mark_.clear();
    h_bulk_ = nullptr; h_bulk_cap_ = 0; bulk_busy_ = false;
    h_stage_vals_ = nullptr; h_stage_addr_ = nullptr; h_stage_index_ = nullptr;
    h_irec_ = nullptr; h_out_ = nullptr; h_nb_off_ = nullptr; h_nb_count_ = nullptr;
    h_ieps2_ = nullptr; d_ieps2_ = nullptr; h_energy_ = nullptr; d_energy_ = nullptr;
    ev_stage_ = ev_begin_ = ev_pred0_ = ev_pred1_ = ev_force0_ = ev_force1_ = ev_done_ = nullptr;
    stream_ = nullptr;
    cap_ = 0; call_cap_ = 0; part_cap_ = 0; nb_alloc_ = 0;
    n_staged_ = 0; slot_of_.clear(); nonident_.clear(); n_nonident_ = 0;
    pred_valid_ = pred64_valid_ = false; pending_ = false; xmax_ = 0; E_ = -1000;
    open_ = false;
}

int Engine::reset() {
    if (!open_) return 0;
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    cudaGetLastError();  // clear a sticky non-fatal error, if any
    if (d_tile_cnt_) {
        cudaMemsetAsync(d_tile_cnt_, 0, sizeof(int) * call_cap_, stream_);
        cudaStreamSynchronize(stream_);
    }
    if (d_out_) {
        cudaMemsetAsync(d_out_, 0, 16, stream_);
        cudaStreamSynchronize(stream_);
    }
    small_parity_ = 0;
    for (int k = 0; k < n_staged_; ++k) slot_of_[h_stage_addr_[k]] = -1;
    n_staged_ = 0;
    pending_ = false;
    pred_valid_ = pred64_valid_ = false;
    last_error.clear();
    return 0;
}

int Engine::set_npipes(int np) {
    if (np < 1) return -1;
    npipes_ = np;
    return 0;
}

int Engine::set_mode(int mode) {
    if (mode != kModeF64 && mode != kModeMixed) return -1;
    if (mode != mode_) pred_valid_ = false;
    mode_ = mode;
    return 0;
}

int Engine::ensure_capacity(int address) {
    if (address < cap_) return 0;
    int ncap = std::max(cap_ * 2, round_up(address + 1, kPadTile));
    ncap = round_up(ncap, kPadTile);
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    G6_CHECK(cudaStreamSynchronize(stream_), "sync");
    double *nraw = nullptr;
    int *nidx = nullptr;
    void *nrec = nullptr;
    G6_CHECK(cudaMalloc(&nraw, sizeof(double) * JF_COUNT * (size_t)ncap), "j-memory");
    G6_CHECK(cudaMalloc(&nidx, sizeof(int) * (size_t)ncap), "j-memory");
    G6_CHECK(cudaMalloc(&nrec, (size_t)kRecMax * ncap), "j-records");
    G6_CHECK(cudaMemsetAsync(nraw, 0, sizeof(double) * JF_COUNT * (size_t)ncap, stream_), "memset");
    G6_CHECK(cudaMemsetAsync(nidx, 0xff, sizeof(int) * (size_t)ncap, stream_), "memset");
    if (cap_ > 0) {
        G6_CHECK(cudaMemcpy2DAsync(nraw, sizeof(double) * ncap, d_jraw_, sizeof(double) * cap_,
                                   sizeof(double) * cap_, JF_COUNT, cudaMemcpyDeviceToDevice, stream_),
                 "grow copy");
        G6_CHECK(cudaMemcpyAsync(nidx, d_jindex_, sizeof(int) * cap_, cudaMemcpyDeviceToDevice, stream_),
                 "grow copy");
    }
    G6_CHECK(cudaStreamSynchronize(stream_), "sync");
    if (d_jraw_) cudaFree(d_jraw_);
    if (d_jindex_) cudaFree(d_jindex_);
    if (d_jrec_) cudaFree(d_jrec_);
    d_jraw_ = nraw;
    d_jindex_ = nidx;
    d_jrec_ = nrec;
    cap_ = ncap;
    slot_of_.resize(cap_, -1);
    nonident_.resize(cap_, 0);
    pred_valid_ = pred64_valid_ = false;
    return 0;
}

int Engine::set_j(int address, int index, double tj, double mass, const double *k18,
                  const double *j6, const double *a2, const double *v, const double *x) {
    if (address < 0) {
        last_error = "g6b200: negative j address";
        return -1;
    }
    if (!open_ && open(env_int("G6B200_DEVICE", 0), 0)) return -1;
    if (ensure_capacity(address)) return -1;
    if (stage_busy_) {
        G6_CHECK(cudaEventSynchronize(ev_stage_), "stage wait");
        stage_busy_ = false;
    }
    int slot = slot_of_[address];
    if (slot < 0) {
        if (n_staged_ == stage_cap_) {
            if (flush_j()) return -1;
            G6_CHECK(cudaEventSynchronize(ev_stage_), "stage wait");
            stage_busy_ = false;
        }
        slot = n_staged_++;
        slot_of_[address] = slot;
        h_stage_addr_[slot] = address;
    }
    h_stage_index_[slot] = index;
    double *r = h_stage_vals_ + (size_t)slot * JF_COUNT;
    r[JF_T] = tj;
    r[JF_M] = mass;
    for (int c = 0; c < 3; ++c) {
        r[JF_X + c] = x[c];
        r[JF_V + c] = v[c];
        r[JF_A2 + c] = a2[c];
        r[JF_J6 + c] = j6[c];
        r[JF_K18 + c] = k18 ? k18[c] : 0.0;
        double ax = std::fabs(x[c]);
        if (ax > xmax_) xmax_ = ax;
    }
    bool ni = address != index;
    if (ni != (bool)nonident_[address]) {
        nonident_[address] = ni;
        n_nonident_ += ni ? 1 : -1;
    }
    stats_.j_updates++;
    return 0;
}

int Engine::flush_j() {
    if (!open_ || n_staged_ == 0) return 0;
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    const int n = n_staged_;
    G6_CHECK(cudaMemcpyAsync(d_stage_vals_, h_stage_vals_, sizeof(double) * JF_COUNT * n,
                             cudaMemcpyHostToDevice, stream_), "stage copy");
    G6_CHECK(cudaMemcpyAsync(d_stage_addr_, h_stage_addr_, sizeof(int) * n, cudaMemcpyHostToDevice, stream_),
             "stage copy");
    G6_CHECK(cudaMemcpyAsync(d_stage_index_, h_stage_index_, sizeof(int) * n, cudaMemcpyHostToDevice, stream_),
             "stage copy");
    launch_scatter(stream_, n, d_stage_addr_, d_stage_index_, d_stage_vals_, d_jraw_, d_jindex_, cap_);
    G6_CHECK(cudaGetLastError(), "scatter launch");
    G6_CHECK(cudaEventRecord(ev_stage_, stream_), "event");
    stage_busy_ = true;
    stats_.h2d_bytes += (long long)n * (JF_COUNT * 8 + 8);
    for (int k = 0; k < n; ++k) slot_of_[h_stage_addr_[k]] = -1;
    n_staged_ = 0;
    pred_valid_ = pred64_valid_ = false;
    return 0;
}

int Engine::set_j_bulk(int n, const int *address, const int *index, const double *tj, const double *mass,
                       const double *k18, const double *j6, const double *a2, const double *v, const double *x) {
    auto one_by_one = [&]() {
        for (int k = 0; k < n; ++k) {
            const int a = address ? address[k] : k;
            if (set_j(a, index ? index[k] : a, tj[k], mass[k], k18 ? k18 + 3 * (size_t)k : nullptr,
                      j6 + 3 * (size_t)k, a2 + 3 * (size_t)k, v + 3 * (size_t)k, x + 3 * (size_t)k))
                return -1;
        }
        return 0;
    };
    constexpr int kBulkMin = 4096;
    if (n <= 0) return 0;
    if (n < kBulkMin) return one_by_one();
    if (!open_ && open(env_int("G6B200_DEVICE", 0), 0)) return -1;
    int amax = n - 1;
    if (address) {
        amax = -1;
        for (int k = 0; k < n; ++k) {
            if (address[k] < 0) {
                last_error = "g6b200: negative j address";
                return -1;
            }
            amax = std::max(amax, address[k]);
        }
        if ((size_t)amax + 1 > bulk_mark_.size()) bulk_mark_.resize((size_t)amax + 1, 0);
        if (++bulk_gen_ == 0) {
            std::fill(bulk_mark_.begin(), bulk_mark_.end(), 0u);
            bulk_gen_ = 1;
        }
        for (int k = 0; k < n; ++k) {
            if (bulk_mark_[address[k]] == bulk_gen_) return one_by_one();  // repeated address: last write wins
            bulk_mark_[address[k]] = bulk_gen_;
        }
    }
    if (ensure_capacity(amax)) return -1;
    if (flush_j()) return -1;  // earlier single updates land first
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    const size_t nd = (size_t)n, vec = 24 * nd;
    const size_t bytes = 16 * nd + 5 * vec + 8 * nd + 9 * 16;  // nine arrays, each start 16-byte aligned
    if (bytes > bulk_cap_) {
        G6_CHECK(cudaStreamSynchronize(stream_), "sync");
        if (d_bulk_) cudaFree(d_bulk_);
        d_bulk_ = nullptr;
        bulk_cap_ = 0;
        G6_CHECK(cudaMalloc(&d_bulk_, bytes), "bulk j");
        bulk_cap_ = bytes;
    }
    // The caller's arrays are gathered into one pinned block by a few host
    // threads (and max |x| taken on the way), then sent in one copy.
    if (bytes > h_bulk_cap_) {
        if (h_bulk_) {
            G6_CHECK(cudaEventSynchronize(ev_stage_), "bulk wait");
            cudaFreeHost(h_bulk_);
        }
        h_bulk_ = nullptr;
        h_bulk_cap_ = 0;
        G6_CHECK(cudaMallocHost(&h_bulk_, bytes), "pinned bulk j");
        h_bulk_cap_ = bytes;
    } else if (bulk_busy_) {
        G6_CHECK(cudaEventSynchronize(ev_stage_), "bulk wait");  // the previous bulk copy read h_bulk_
    }
    struct Part {
        const void *src;
        size_t bytes, off;
    };
    Part parts[9];
    int np = 0;
    size_t off = 0;
    auto add = [&](const void *src, size_t b) -> const void * {
        if (!src) return nullptr;
        parts[np++] = {src, b, off};
        const void *d = d_bulk_ + off;
        off += (b + 15) / 16 * 16;
        return d;
    };
    BulkJ b;
    b.t = static_cast<const double *>(add(tj, 8 * nd));
    b.m = static_cast<const double *>(add(mass, 8 * nd));
    b.x = static_cast<const double *>(add(x, vec));
    b.v = static_cast<const double *>(add(v, vec));
    b.a2 = static_cast<const double *>(add(a2, vec));
    b.j6 = static_cast<const double *>(add(j6, vec));
    b.k18 = static_cast<const double *>(add(k18, vec));
    b.addr = static_cast<const int *>(add(address, 4 * nd));
    b.index = static_cast<const int *>(add(index, 4 * nd));
    double tmax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    parallel_ranges(nd, 16384, [&](size_t lo, size_t hi, size_t t) {
        for (int k = 0; k < np; ++k) {
            const size_t per = parts[k].bytes / nd;  // bytes per particle of this array
            memcpy(h_bulk_ + parts[k].off + lo * per, static_cast<const unsigned char *>(parts[k].src) + lo * per,
                   (hi - lo) * per);
        }
        double m = 0;
        for (size_t q = 3 * lo; q < 3 * hi; ++q) m = std::max(m, std::fabs(x[q]));
        tmax[t] = m;
    });
    G6_CHECK(cudaMemcpyAsync(d_bulk_, h_bulk_, off, cudaMemcpyHostToDevice, stream_), "bulk j copy");
    G6_CHECK(cudaEventRecord(ev_stage_, stream_), "event");
    bulk_busy_ = true;
    launch_scatter_bulk(stream_, n, b, d_jraw_, d_jindex_, cap_);
    G6_CHECK(cudaGetLastError(), "bulk scatter launch");
    stats_.launches++;
    stats_.h2d_bytes += (long long)off;
    stats_.j_updates += n;
    double xm = xmax_;
    for (double m : tmax) xm = std::max(xm, m);
    xmax_ = xm;
    for (int k = 0; k < n; ++k) {
        const int a = address ? address[k] : k;
        const bool ni = index && index[k] != a;
        if (ni != (bool)nonident_[a]) {
            nonident_[a] = ni;
            n_nonident_ += ni ? 1 : -1;
        }
    }
    pred_valid_ = pred64_valid_ = false;
    return 0;
}

int Engine::choose_E(double xmax) const {
    if (!(xmax > 0) || !std::isfinite(xmax)) return 1;
    int e = std::ilogb(xmax) + 2;  // xmax < 2^(E-1): a factor-2 margin
    return std::max(e, -60);
}

FixedScale Engine::scale() const {
    FixedScale fs;
    fs.to_units = std::ldexp(1.0, 23 - E_);
    fs.hi_unit = std::ldexp(1.0, E_ - 23);
    fs.lo_unit = std::ldexp(1.0, E_ - 46);
    return fs;
}

int Engine::ensure_call_buffers(int ni, bool nb, size_t part_bytes) {
    if (ni > call_cap_ || part_bytes > part_cap_ || (nb && nb_alloc_ < std::max(call_cap_, ni))) stats_.grows++;
    if (ni > call_cap_) {
        int ncap = std::max(ni, npipes_);
        if (h_irec_) cudaFreeHost(h_irec_);
        if (d_irec_) cudaFree(d_irec_);
        if (h_out_) cudaFreeHost(h_out_);
        if (d_out_) cudaFree(d_out_);
        if (h_ieps2_) cudaFreeHost(h_ieps2_);
        if (d_ieps2_) cudaFree(d_ieps2_);
        h_irec_ = d_irec_ = nullptr;
        h_out_ = d_out_ = nullptr;
        h_ieps2_ = d_ieps2_ = nullptr;
        OutLayout L(ncap);
        G6_CHECK(cudaMallocHost(&h_irec_, sizeof(IRec) * ncap), "pinned i");
        G6_CHECK(cudaMalloc(&d_irec_, sizeof(IRec) * ncap), "i-records");
        G6_CHECK(cudaMallocHost(&h_ieps2_, sizeof(double) * ncap), "pinned i");
        G6_CHECK(cudaMalloc(&d_ieps2_, sizeof(double) * ncap), "i-softening");
        G6_CHECK(cudaMallocHost(&h_out_, L.total), "pinned out");
        G6_CHECK(cudaMalloc(&d_out_, L.total), "out");
        if (d_tile_cnt_) cudaFree(d_tile_cnt_);
        d_tile_cnt_ = nullptr;
        G6_CHECK(cudaMalloc(&d_tile_cnt_, sizeof(int) * ncap), "tile counters");
        G6_CHECK(cudaMemsetAsync(d_tile_cnt_, 0, sizeof(int) * ncap, stream_), "memset");
        G6_CHECK(cudaMemsetAsync(d_out_, 0, 16, stream_), "memset");  // both status words clear
        small_parity_ = 0;
        call_cap_ = ncap;
    }
    if (part_bytes > part_cap_) {
        if (d_part_) cudaFree(d_part_);
        d_part_ = nullptr;
        size_t nb_ = part_bytes + part_bytes / 4;
        G6_CHECK(cudaMalloc(&d_part_, nb_), "partials");
        part_cap_ = nb_;
    }
    if (nb && nb_alloc_ < call_cap_) {
        if (d_nb_count_) cudaFree(d_nb_count_);
        if (d_nb_list_) cudaFree(d_nb_list_);
        if (d_nb_sorted_) cudaFree(d_nb_sorted_);
        if (d_nb_off_) cudaFree(d_nb_off_);
        if (h_nb_off_) cudaFreeHost(h_nb_off_);
        if (h_nb_count_) cudaFreeHost(h_nb_count_);
        const int n = call_cap_;
        G6_CHECK(cudaMalloc(&d_nb_count_, sizeof(int) * n), "nb");
        G6_CHECK(cudaMalloc(&d_nb_list_, sizeof(int) * (size_t)n * nb_cap_), "nb");
        G6_CHECK(cudaMalloc(&d_nb_sorted_, sizeof(int) * (size_t)n * nb_cap_), "nb");
        G6_CHECK(cudaMalloc(&d_nb_off_, sizeof(long long) * (n + 1)), "nb");
        G6_CHECK(cudaMallocHost(&h_nb_off_, sizeof(long long) * (n + 1)), "nb");
        G6_CHECK(cudaMallocHost(&h_nb_count_, sizeof(int) * n), "nb");
        nb_alloc_ = n;
    }
    return 0;
}

// Buffers of the mixed mode's FP64 refinement for calls of up to ni i (and
// FP64 j-records for the j-memory's capacity).
int Engine::ensure_refine_buffers(int ni) {
    if (ni > ref_cap_) {
        const int n = std::max(ni, npipes_);
        auto dfree = [](void *p) { if (p) cudaFree(p); };
        dfree(d_q_); dfree(d_ref_list_); dfree(d_ref_tcnt_); dfree(d_ref_irec_); dfree(d_ref_part_);
        d_q_ = nullptr; d_ref_list_ = d_ref_tcnt_ = nullptr; d_ref_irec_ = nullptr; d_ref_part_ = nullptr;
        ref_cap_ = 0;
        G6_CHECK(cudaMalloc(&d_q_, sizeof(float) * 2 * (size_t)n), "refine");
        G6_CHECK(cudaMalloc(&d_ref_list_, sizeof(int) * (size_t)n), "refine");
        G6_CHECK(cudaMalloc(&d_ref_tcnt_, sizeof(int) * (size_t)n), "refine");
        G6_CHECK(cudaMemsetAsync(d_ref_tcnt_, 0, sizeof(int) * (size_t)n, stream_), "refine");
        G6_CHECK(cudaMalloc(&d_ref_irec_, sizeof(IRec) * (size_t)n), "refine");
        G6_CHECK(cudaMalloc(&d_ref_part_, sizeof(Partial) * refine_partial_records(n)), "refine");
        ref_cap_ = n;
        stats_.grows++;
    }
    return ensure_jrec64();
}

int Engine::firsthalf(int nj, int ni, const int *index, const double (*xi)[3], const double (*vi)[3],
                      double eps2, const double *h2) {
    return firsthalf_impl(nj, ni, index, xi, vi, eps2, nullptr, h2);
}

int Engine::firsthalf_g4(int nj, int ni, const double (*xi)[3], const double (*vi)[3], const double *eps2,
                         const double *h2) {
    if (mode_ != kModeF64) {
        call_error_ = true;
        last_error = "g6b200: the GRAPE-4 pipeline runs in FP64 mode only";
        return -1;
    }
    return firsthalf_impl(nj, ni, nullptr, xi, vi, 0.0, eps2, h2);
}

int Engine::firsthalf_impl(int nj, int ni, const int *index, const double (*xi)[3], const double (*vi)[3],
                           double eps2, const double *ieps2, const double *h2) {
    const auto h0 = std::chrono::steady_clock::now();
    struct HostTimer {
        EngineStats &st;
        std::chrono::steady_clock::time_point t0;
        ~HostTimer() {
            st.host_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    } host_timer{stats_, h0};
    call_error_ = false;
    if (!open_ && open(env_int("G6B200_DEVICE", 0), 0)) {
        call_error_ = true;
        return -1;
    }
    if (ni < 0 || nj < 0 || ni > npipes_) {
        char buf[128];
        snprintf(buf, sizeof buf, "g6b200: bad call sizes ni=%d nj=%d (npipes=%d)", ni, nj, npipes_);
        last_error = buf;
        call_error_ = true;
        return -1;
    }
    if (cudaSetDevice(device_) != cudaSuccess) {
        call_error_ = true;
        return fail("cudaSetDevice", cudaErrorInvalidDevice);
    }
    if (nj > 0 && ensure_capacity(nj - 1)) {
        call_error_ = true;
        return -1;
    }
    bool nb = false;
    for (int i = 0; i < ni; ++i) {
        double hh = h2 ? h2[i] : default_h2_;
        if (hh > 0) nb = true;
    }
    if (ensure_call_buffers(ni, nb, 0)) {
        call_error_ = true;
        return -1;
    }
    double tmax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    parallel_ranges((size_t)ni, 65536, [&](size_t lo, size_t hi, size_t t) {
        double xm = 0;
        for (size_t i = lo; i < hi; ++i) {
            IRec &r = h_irec_[i];
            for (int c = 0; c < 3; ++c) {
                r.x[c] = xi[i][c];
                r.v[c] = vi[i][c];
                xm = std::max(xm, std::fabs(xi[i][c]));
            }
            r.h2 = h2 ? h2[i] : default_h2_;
            r.index = index ? index[i] : -1;
            r.pad = 0;
            if (ieps2) h_ieps2_[i] = ieps2[i];
        }
        tmax[t] = xm;
    });
    double xm = xmax_;
    for (double m : tmax) xm = std::max(xm, m);
    xmax_ = xm;
    if (ni == 2 && index && index[0] == index[1]) stats_.pair_calls++;
    call_ni_ = ni;
    call_nj_ = nj;
    call_eps2_ = eps2;
    call_nb_ = nb;
    call_g4_ = ieps2 != nullptr;
    call_sweep_ = false;
    call_pot_ = pot_request_;
    call_energy_ = false;
    call_split_ = split_request_;
    call_copy_ = call_split_ == 0;  // a split call's results stay on the device
    call_i0_ = 0;
    nb_read_ = false;
    // The one-launch form pays for its 14 KB parameter block by replacing the
    // staged updates' copies and scatter: without updates the copy path
    // (status clear, prediction, i-record copy) is as fast.
    call_small_ = small_enabled_ && n_staged_ > 0 && ni <= kSmallMax && n_staged_ <= kSmallMax;
    if (!call_small_ && flush_j()) {
        call_error_ = true;
        return -1;
    }
    int rc = launch_call();
    if (rc) {
        call_error_ = true;
        return rc;
    }
    pending_ = true;
    return 0;
}

// Record that the j-records of layout km (the mixed ones in d_jrec_, or the
// FP64 ones in d_jrec64_ when the engine is in mixed mode) hold the current
// j-state at the block time.
void Engine::mark_predicted(int nj, int km) {
    if (mode_ == kModeMixed && km == kKernF64) {
        pred64_valid_ = true;
        pred64_ti_ = ti_;
        pred64_nj_ = nj;
        return;
    }
    pred_valid_ = true;
    pred_ti_ = ti_;
    pred_nj_ = nj;
    pred_mode_ = km;
    pred_E_ = E_;
}

// FP64 j-records beside the mixed ones (the refinement and the FP64 small
// calls of the mixed mode), for the j-memory's capacity.
int Engine::ensure_jrec64() {
    if (jrec64_cap_ >= cap_) return 0;
    if (d_jrec64_) cudaFree(d_jrec64_);
    d_jrec64_ = nullptr;
    jrec64_cap_ = 0;
    G6_CHECK(cudaMalloc(&d_jrec64_, sizeof(JRecF64) * (size_t)cap_), "FP64 records");
    jrec64_cap_ = cap_;
    pred64_valid_ = false;
    return 0;
}

int Engine::launch_call() {
    const int ni = call_ni_, nj = call_nj_;
    call_refine_ = false;
    // Mixed mode: a call of fewer than mixed_min_work_ interactions runs in
    // FP64 on the FP64 j-records (d_jrec64_, kept beside the mixed ones):
    // such calls are latency-bound, so FP64 costs them nothing, and they get
    // FP64 results (kira's small blocks at its tiny first steps among them).
    call_f64_ = mode_ == kModeMixed && mixed_min_work_ > 0 && !call_g4_ && !call_split_ && !call_sweep_ &&
                !call_pot_ && !call_energy_ && (long long)ni * round_up(nj, tile_size(kmode())) < mixed_min_work_;
    const int km = call_f64_ ? kKernF64 : kmode();
    const int T = tile_size(km);
    const int nj_pad = round_up(nj, T);
    if (nj_pad > cap_ && ensure_capacity(nj_pad - 1)) return -1;
    if (call_f64_ && ensure_jrec64()) return -1;
    int E = std::max(E_, choose_E(xmax_));
    if (E != E_) {
        E_ = E;
        pred_valid_ = false;
    }
    const FixedScale fs = scale();
    OutLayout L(ni);
    timed_ = event_timing_ || call_sweep_;
    if (timed_) G6_CHECK(cudaEventRecord(ev_begin_, stream_), "event");
    const bool small = call_small_ && !call_sweep_;
    unsigned *status2 = reinterpret_cast<unsigned *>(d_out_ + L.status);
    if (small) {
        call_parity_ = small_parity_;
        small_parity_ ^= 1;
    } else {
        G6_CHECK(cudaMemsetAsync(d_out_, 0, 16, stream_), "memset");
        call_parity_ = 0;
        small_parity_ = 1;  // word 1 stays clear: this call reports into word 0
    }
    unsigned *status = status2 + call_parity_;
    pred_timed_ = false;
    const bool staged = small && n_staged_ > 0;
    bool need_pred;
    if (call_f64_) {
        need_pred = !pred64_valid_ || pred64_ti_ != ti_ || pred64_nj_ != nj || staged;
        if (staged) pred_valid_ = v2_valid_ = false;  // the updates land in the raw j-state: the mixed records are stale
    } else {
        need_pred = !pred_valid_ || pred_ti_ != ti_ || pred_nj_ != nj || pred_mode_ != km || pred_E_ != E_ || staged;
        if (need_pred) pred64_valid_ = v2_valid_ = false;  // the FP64 records and |v| scale follow
    }
    void *jrec = call_f64_ ? d_jrec64_ : d_jrec_;
    // FP64 records are predicted over the mixed layout's padding too (the
    // refinement reads them with the same nj).
    const int pred_pad = call_f64_ ? round_up(nj, tile_size(kmode())) : nj_pad;
    if (small) {
        // Updates, prediction and i-records in one launch whose parameter is
        // the call's host data (no host->device copy).
        SmallCall &sc = small_call_;
        sc.n_upd = n_staged_;
        sc.ni = ni;
        sc.nj = nj;
        sc.nj_pad = pred_pad;
        sc.cap = cap_;
        sc.predict = need_pred;
        sc.parity = call_parity_;
        sc.g4 = call_g4_;
        sc.ti = ti_;
        sc.fs = fs;
        int order[kSmallMax];
        for (int k = 0; k < n_staged_; ++k) order[k] = k;
        std::sort(order, order + n_staged_, [&](int a, int b) { return h_stage_addr_[a] < h_stage_addr_[b]; });
        for (int k = 0; k < n_staged_; ++k) {
            const int sl = order[k];
            sc.addr[k] = h_stage_addr_[sl];
            sc.index[k] = h_stage_index_[sl];
            memcpy(sc.vals[k], h_stage_vals_ + (size_t)sl * JF_COUNT, sizeof(double) * JF_COUNT);
            slot_of_[h_stage_addr_[sl]] = -1;
        }
        memcpy(sc.irec, h_irec_, sizeof(IRec) * ni);
        if (call_g4_) memcpy(sc.ieps2, h_ieps2_, sizeof(double) * ni);
        stats_.h2d_bytes += (long long)sizeof(SmallCall);
        n_staged_ = 0;
        if (timed_) G6_CHECK(cudaEventRecord(ev_pred0_, stream_), "event");
        launch_small_call(stream_, km, sc, d_jraw_, d_jindex_, jrec, d_irec_, d_ieps2_, status2);
        G6_CHECK(cudaGetLastError(), "small call launch");
        stats_.launches++;
        if (timed_) G6_CHECK(cudaEventRecord(ev_pred1_, stream_), "event");
        pred_timed_ = need_pred;
        if (need_pred) {
            stats_.predictions++;
            mark_predicted(nj, km);
        }
    } else if (need_pred) {
        if (timed_) G6_CHECK(cudaEventRecord(ev_pred0_, stream_), "event");
        launch_predict(stream_, km, d_jraw_, d_jindex_, cap_, nj, pred_pad, ti_, fs, jrec, status);
        G6_CHECK(cudaGetLastError(), "predict launch");
        stats_.launches++;
        if (timed_) G6_CHECK(cudaEventRecord(ev_pred1_, stream_), "event");
        stats_.predictions++;
        pred_timed_ = true;
        mark_predicted(nj, km);
    }
    if (ni > 0) {
        if (small) {
            // i-records (and softening) written by the small-call launch
        } else if (call_sweep_) {
            launch_irec_from_j(stream_, d_jraw_, d_jindex_, cap_, call_i0_, ni, ti_, d_irec_);
            G6_CHECK(cudaGetLastError(), "i-record launch");
            stats_.launches++;
        } else {
            G6_CHECK(cudaMemcpyAsync(d_irec_, h_irec_, sizeof(IRec) * ni, cudaMemcpyHostToDevice, stream_),
                     "i copy");
            stats_.h2d_bytes += (long long)sizeof(IRec) * ni;
            if (call_g4_) {
                G6_CHECK(cudaMemcpyAsync(d_ieps2_, h_ieps2_, sizeof(double) * ni, cudaMemcpyHostToDevice, stream_),
                         "i copy");
                stats_.h2d_bytes += (long long)sizeof(double) * ni;
            }
        }
        ForceConfig cfg = override_.il > 0 ? override_ : choose_config(km, ni, nj_pad, num_sms_, call_nb_);
        // Potential-only kernel (one i per thread) for the paired mixed and
        // FP64 layouts; the scalar mixed layout runs its full kernel.
        const bool pot_k = call_pot_ && km != kKernMixedDS;
        if (pot_k) cfg.r = 1;
        // Mixed mode (paired layout): ill-conditioned particles are
        // recomputed in FP64 (refine.cu); not for potential-only, j-split
        // or GRAPE-4 calls.
        call_refine_ = refine_enabled_ && km == kKernMixedP && !pot_k && !call_split_ && !call_g4_;
        if (call_refine_ && ensure_refine_buffers(ni)) return -1;
        if (call_split_) cfg.jper = call_split_;
        if (ensure_call_buffers(ni, call_nb_, call_split_ ? partial_bytes_fixed(call_split_, nj_pad, ni)
                                                          : partial_bytes(cfg, ni)))
            return -1;
        last_cfg_ = cfg;
        ForceParams p{};
        p.jrec = jrec;
        p.nj = nj;
        p.nj_pad = nj_pad;
        p.irec = d_irec_;
        p.ni = ni;
        p.eps2 = call_eps2_;
        p.fs = fs;
        p.part = d_part_;
        p.out_acc = reinterpret_cast<double *>(d_out_ + L.acc);
        p.out_jerk = reinterpret_cast<double *>(d_out_ + L.jerk);
        p.out_pot = reinterpret_cast<double *>(d_out_ + L.pot);
        p.out_nn = reinterpret_cast<int *>(d_out_ + L.nn);
        p.nb_count = d_nb_count_;
        p.nb_list = d_nb_list_;
        p.nb_cap = nb_cap_;
        p.include_self = npipes_ > 48;
        p.status = status;
        p.tile_counter = call_split_ ? nullptr : d_tile_cnt_;
        p.ieps2 = call_g4_ ? d_ieps2_ : nullptr;
        p.keep_partials = call_split_ ? 1 : 0;
        p.out_q = call_refine_ ? d_q_ : nullptr;
        if (call_nb_) G6_CHECK(cudaMemsetAsync(d_nb_count_, 0, sizeof(int) * ni, stream_), "memset");
        if (timed_) G6_CHECK(cudaEventRecord(ev_force0_, stream_), "event");
        G6_CHECK(launch_force(stream_, km, cfg, p, n_nonident_ == 0 && !call_g4_, call_nb_, call_g4_, pot_k),
                 "force launch");
        if (timed_) G6_CHECK(cudaEventRecord(ev_force1_, stream_), "event");
        stats_.launches += 1;
        if (call_refine_) {
            if (!v2_valid_) {
                launch_refine_v2(stream_, d_jraw_, cap_, nj, d_v2_);
                G6_CHECK(cudaGetLastError(), "refine launch");
                stats_.launches += 2;
                v2_valid_ = true;
            }
            if (!pred64_valid_ || pred64_ti_ != ti_ || pred64_nj_ != nj) {
                launch_predict(stream_, kKernF64, d_jraw_, d_jindex_, cap_, nj, nj_pad, ti_, fs, d_jrec64_, status);
                G6_CHECK(cudaGetLastError(), "refine predict launch");
                stats_.launches++;
                mark_predicted(nj, kKernF64);
            }
            RefineArgs ra{};
            ra.ni = ni;
            ra.nj = nj;
            ra.nj_pad = round_up(nj, tile_size(kKernF64));
            ra.ident = n_nonident_ == 0;
            ra.eps2 = call_eps2_;
            ra.v2 = d_v2_;
            ra.q = d_q_;
            ra.irec = d_irec_;
            ra.jrec64 = d_jrec64_;
            ra.acc = p.out_acc;
            ra.jerk = p.out_jerk;
            ra.pot = p.out_pot;
            ra.nn = p.out_nn;
            ra.count = d_ref_small_;
            ra.counter = d_ref_small_ + 1;
            ra.pre = d_ref_small_ + 2;
            ra.done = reinterpret_cast<unsigned *>(d_ref_small_ + 6);
            ra.list = d_ref_list_;
            ra.irec_ref = d_ref_irec_;
            ra.part = d_ref_part_;
            ra.tcnt = d_ref_tcnt_;
            ra.items = d_ref_items_;
            ra.status = status;
            G6_CHECK(launch_refine(stream_, ra, num_sms_), "refine launch");
            stats_.launches += 2;
            G6_CHECK(cudaMemcpyAsync(h_ref_count_, d_ref_small_ + 5, sizeof(int), cudaMemcpyDeviceToHost, stream_),
                     "refine count");
        }
        if (call_split_) {
            split_nsplit_ = std::max(1, (nj_pad + call_split_ - 1) / call_split_);
            launch_split_agree(stream_, ni, split_nsplit_, d_part_, split_agree_);
            G6_CHECK(cudaGetLastError(), "split launch");
            stats_.launches++;
        }
        if (call_energy_) {
            launch_energy(stream_, ni, call_i0_, d_irec_, d_jraw_, cap_, p.out_pot, d_energy_);
            G6_CHECK(cudaGetLastError(), "energy launch");
            stats_.launches += 2;
            G6_CHECK(cudaMemcpyAsync(h_energy_, d_energy_ + 2 * kEnergyBlocks, 2 * sizeof(double),
                                     cudaMemcpyDeviceToHost, stream_), "energy copy");
            stats_.d2h_bytes += 2 * (long long)sizeof(double);
        }
        if (call_nb_) {
            stats_.nb_calls++;
            G6_CHECK(launch_nb_compact(stream_, ni, d_nb_count_, d_nb_list_, nb_cap_, d_nb_off_, d_nb_sorted_),
                     "nb compact");
            stats_.launches += 2;
            G6_CHECK(cudaMemcpyAsync(h_nb_off_, d_nb_off_, sizeof(long long) * (ni + 1), cudaMemcpyDeviceToHost,
                                     stream_), "nb copy");
            G6_CHECK(cudaMemcpyAsync(h_nb_count_, d_nb_count_, sizeof(int) * ni, cudaMemcpyDeviceToHost, stream_),
                     "nb copy");
        }
    } else if (timed_) {
        G6_CHECK(cudaEventRecord(ev_force0_, stream_), "event");
        G6_CHECK(cudaEventRecord(ev_force1_, stream_), "event");
    }
    const size_t out_bytes = call_copy_ ? L.total : L.acc;  // status header only when not copying
    G6_CHECK(cudaMemcpyAsync(h_out_, d_out_, out_bytes, cudaMemcpyDeviceToHost, stream_), "out copy");
    stats_.d2h_bytes += (long long)out_bytes;
    G6_CHECK(cudaEventRecord(ev_done_, stream_), "event");
    stats_.calls++;
    stats_.interactions += (long long)ni * nj;
    return 0;
}

int Engine::lasthalf(int ni, double (*acc)[3], double (*jerk)[3], double *pot, int *nn) {
    if (call_error_ || !pending_) {
        pending_ = false;
        if (last_error.empty()) last_error = "g6b200: lasthalf without a successful firsthalf";
        return 1;
    }
    pending_ = false;
    int rc = wait_call();
    if (rc) return rc;
    const int n = std::min(ni, call_ni_);
    OutLayout L(call_ni_);
    parallel_ranges((size_t)n, 65536, [&](size_t lo, size_t hi, size_t) {
        if (acc) memcpy(acc[lo], h_out_ + L.acc + 24 * lo, 24 * (hi - lo));
        if (jerk) memcpy(jerk[lo], h_out_ + L.jerk + 24 * lo, 24 * (hi - lo));
        if (pot) memcpy(pot + lo, h_out_ + L.pot + 8 * lo, 8 * (hi - lo));
        if (nn) memcpy(nn + lo, h_out_ + L.nn + 4 * lo, 4 * (hi - lo));
    });
    ++lasthalf_count_;
    if (fault_lasthalf_at_ >= 0 && lasthalf_count_ == fault_lasthalf_at_) {
        last_error = "g6b200: injected lasthalf failure (G6B200_FAULT_LASTHALF)";
        return 5;
    }
    if (fault_pot_at_ >= 0 && lasthalf_count_ == fault_pot_at_ && pot && n > 0) pot[0] = 1.0;
    return 0;
}

int Engine::wait_call() {
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    for (int attempt = 0;; ++attempt) {
        const auto w0 = std::chrono::steady_clock::now();
        cudaError_t e = cudaEventSynchronize(ev_done_);
        stats_.wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        if (e != cudaSuccess) {
            fail("device execution", e);
            return 2;
        }
        unsigned status = reinterpret_cast<unsigned *>(h_out_)[call_parity_];
        if ((status & ST_RANGE) && attempt < 8) {
            // Fixed-point range exceeded: widen by 4x and recompute.
            stats_.range_retries++;
            E_ += 2;
            pred_valid_ = false;
            if (launch_call()) return 2;
            continue;
        }
        if (status & ST_TMA_TIMEOUT) {
            last_error = "g6b200: j-tile copy wait timed out on the device";
            return 3;
        }
        if (status & ST_RANGE) {
            last_error = "g6b200: positions outside the fixed-point range";
            return 4;
        }
        break;
    }
    if (call_refine_) stats_.refined += *h_ref_count_;
    float ms = 0;
    if (!timed_) {
        stats_.last_force_ms = stats_.last_predict_ms = stats_.last_call_ms = 0;
        return 0;
    }
    if (cudaEventElapsedTime(&ms, ev_force0_, ev_force1_) == cudaSuccess) stats_.last_force_ms = ms;
    if (pred_timed_ && cudaEventElapsedTime(&ms, ev_pred0_, ev_pred1_) == cudaSuccess)
        stats_.last_predict_ms = ms;
    else
        stats_.last_predict_ms = 0;
    if (cudaEventElapsedTime(&ms, ev_begin_, ev_done_) == cudaSuccess) stats_.last_call_ms = ms;
    return 0;
}

int Engine::sweep(int nj, int i0, int ni, double eps2, bool copy_out, double (*acc)[3], double (*jerk)[3],
                  double *pot, int *nn) {
    if (pending_) {
        last_error = "g6b200: sweep while a firsthalf call is pending";
        return -1;
    }
    if (!open_ && open(env_int("G6B200_DEVICE", 0), 0)) return -1;
    if (ni < 0 || nj < 0 || i0 < 0 || i0 + ni > nj) {
        last_error = "g6b200: bad sweep range";
        return -1;
    }
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    if (nj > 0 && ensure_capacity(nj - 1)) return -1;
    if (ensure_call_buffers(ni, false, 0)) return -1;
    call_ni_ = ni;
    call_nj_ = nj;
    call_eps2_ = eps2;
    call_nb_ = false;
    call_g4_ = false;
    call_small_ = false;
    call_sweep_ = true;
    call_pot_ = false;
    call_energy_ = false;
    call_split_ = 0;
    call_copy_ = copy_out;
    call_i0_ = i0;
    nb_read_ = false;
    if (flush_j()) return -1;
    if (launch_call()) return -1;
    int rc = wait_call();
    if (rc) return rc;
    if (copy_out) {
        OutLayout L(ni);
        if (acc) memcpy(acc, h_out_ + L.acc, 24 * (size_t)ni);
        if (jerk) memcpy(jerk, h_out_ + L.jerk, 24 * (size_t)ni);
        if (pot) memcpy(pot, h_out_ + L.pot, 8 * (size_t)ni);
        if (nn) memcpy(nn, h_out_ + L.nn, 4 * (size_t)ni);
    }
    return 0;
}

int Engine::potential(int nj, int ni, const int *index, const double (*xi)[3], double eps2, double *pot) {
    if (pending_) {
        last_error = "g6b200: potential call while a firsthalf call is pending";
        return -1;
    }
    std::vector<double> zv(3 * (size_t)std::max(ni, 1), 0.0);  // the potential needs no velocities
    pot_request_ = true;
    int rc = firsthalf_impl(nj, ni, index, xi, reinterpret_cast<const double (*)[3]>(zv.data()), eps2, nullptr,
                            nullptr);
    pot_request_ = false;
    if (rc) return rc;
    return lasthalf(ni, nullptr, nullptr, pot, nullptr);
}

int Engine::energies(int nj, double eps2, double *epot, double *ekin, double *pot) {
    if (pending_) {
        last_error = "g6b200: energy call while a firsthalf call is pending";
        return -1;
    }
    if (!open_ && open(env_int("G6B200_DEVICE", 0), 0)) return -1;
    if (nj < 0) {
        last_error = "g6b200: bad energy call size";
        return -1;
    }
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    if (nj > 0 && ensure_capacity(nj - 1)) return -1;
    if (ensure_call_buffers(nj, false, 0)) return -1;
    call_ni_ = nj;
    call_nj_ = nj;
    call_eps2_ = eps2;
    call_nb_ = false;
    call_g4_ = false;
    call_small_ = false;
    call_sweep_ = true;
    call_pot_ = true;
    call_energy_ = nj > 0;
    call_split_ = 0;
    call_copy_ = pot != nullptr;
    call_i0_ = 0;
    nb_read_ = false;
    int rc = flush_j() || launch_call() ? -1 : wait_call();
    call_energy_ = false;
    call_pot_ = false;
    if (rc) return rc;
    if (epot) *epot = nj > 0 ? h_energy_[0] : 0.0;
    if (ekin) *ekin = nj > 0 ? h_energy_[1] : 0.0;
    if (pot) memcpy(pot, h_out_ + OutLayout(nj).pot, 8 * (size_t)nj);
    return 0;
}

void Engine::set_position_range(double xmax) {
    if (xmax > xmax_) xmax_ = xmax;
    const int E = std::max(E_, choose_E(xmax_));
    if (E != E_) {
        E_ = E;
        pred_valid_ = false;
    }
}

int Engine::split_begin(int nj, int ni, const int *index, const double (*xi)[3], const double (*vi)[3],
                        double eps2, int block_j, long long *agree, void *stream) {
    if (pending_) {
        last_error = "g6b200: split call while a firsthalf call is pending";
        return -1;
    }
    if (block_j <= 0 || block_j % 256 || !agree) {
        last_error = "g6b200: split call needs block_j a positive multiple of 256 and an agree buffer";
        return -1;
    }
    if (!open_ && open(env_int("G6B200_DEVICE", 0), 0)) return -1;
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    // the caller's earlier work on `agree` comes first
    G6_CHECK(cudaEventRecord(ev_ext_, static_cast<cudaStream_t>(stream)), "event");
    G6_CHECK(cudaStreamWaitEvent(stream_, ev_ext_, 0), "stream wait");
    split_request_ = block_j;
    split_agree_ = agree;
    int rc = firsthalf_impl(nj, ni, index, xi, vi, eps2, nullptr, nullptr);
    split_request_ = 0;
    if (rc) return rc;
    pending_ = false;
    rc = wait_call();  // also retries a fixed-point range report (agree is rewritten)
    call_split_ = 0;
    return rc;
}

int Engine::split_fix(long long nblocks_total, long long j_offset, const long long *agree, long long *sums,
                      long long *negj, void *stream) {
    if (split_nsplit_ <= 0) {
        last_error = "g6b200: split_fix without a split_begin";
        return -1;
    }
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    G6_CHECK(cudaEventRecord(ev_ext_, cs), "event");
    G6_CHECK(cudaStreamWaitEvent(stream_, ev_ext_, 0), "stream wait");
    launch_split_fix(stream_, call_ni_, split_nsplit_, split_log2_blocks(nblocks_total), j_offset, d_part_, agree,
                     sums, negj);
    G6_CHECK(cudaGetLastError(), "split fix launch");
    stats_.launches++;
    G6_CHECK(cudaEventRecord(ev_ext_, stream_), "event");
    G6_CHECK(cudaStreamWaitEvent(cs, ev_ext_, 0), "stream wait");
    return 0;
}

int Engine::split_finish(long long nblocks_total, long long nj_total, const long long *agree, const long long *sums,
                         const long long *negj, void *stream, double (*acc)[3], double (*jerk)[3], double *pot,
                         int *nn) {
    if (split_nsplit_ <= 0) {
        last_error = "g6b200: split_finish without a split_begin";
        return -1;
    }
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    G6_CHECK(cudaEventRecord(ev_ext_, static_cast<cudaStream_t>(stream)), "event");
    G6_CHECK(cudaStreamWaitEvent(stream_, ev_ext_, 0), "stream wait");
    const int ni = call_ni_;
    OutLayout L(ni);
    launch_split_finish(stream_, ni, split_log2_blocks(nblocks_total), nj_total, agree, sums, negj,
                        reinterpret_cast<double *>(d_out_ + L.acc), reinterpret_cast<double *>(d_out_ + L.jerk),
                        reinterpret_cast<double *>(d_out_ + L.pot), reinterpret_cast<int *>(d_out_ + L.nn));
    G6_CHECK(cudaGetLastError(), "split finish launch");
    stats_.launches++;
    G6_CHECK(cudaMemcpyAsync(h_out_ + L.acc, d_out_ + L.acc, L.total - L.acc, cudaMemcpyDeviceToHost, stream_),
             "out copy");
    stats_.d2h_bytes += (long long)(L.total - L.acc);
    G6_CHECK(cudaStreamSynchronize(stream_), "sync");
    split_nsplit_ = 0;
    if (acc) memcpy(acc, h_out_ + L.acc, 24 * (size_t)ni);
    if (jerk) memcpy(jerk, h_out_ + L.jerk, 24 * (size_t)ni);
    if (pot) memcpy(pot, h_out_ + L.pot, 8 * (size_t)ni);
    if (nn) memcpy(nn, h_out_ + L.nn, 4 * (size_t)ni);
    return 0;
}

int Engine::selftest_copy_timeout(double limit_ms) {
    if (!open_ && open(env_int("G6B200_DEVICE", 0), 0)) return -1;
    if (pending_) {
        last_error = "g6b200: self-test while a firsthalf call is pending";
        return -1;
    }
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    if (ensure_call_buffers(1, false, 0)) return -1;
    G6_CHECK(cudaMemsetAsync(d_out_, 0, 16, stream_), "memset");
    call_parity_ = 0;
    timed_ = false;
    launch_copy_wait_selftest(stream_, reinterpret_cast<unsigned *>(d_out_),
                              (unsigned long long)(limit_ms > 0 ? limit_ms * 1e6 : 1e6));
    G6_CHECK(cudaGetLastError(), "self-test launch");
    G6_CHECK(cudaMemcpyAsync(h_out_, d_out_, 16, cudaMemcpyDeviceToHost, stream_), "status copy");
    G6_CHECK(cudaEventRecord(ev_done_, stream_), "event");
    const int rc = wait_call();
    // both status words clear again for the next call, as after reset()
    G6_CHECK(cudaMemsetAsync(d_out_, 0, 16, stream_), "memset");
    G6_CHECK(cudaStreamSynchronize(stream_), "sync");
    small_parity_ = 0;
    return rc;
}

size_t Engine::footprint_bytes() const {
    return (size_t)cap_ * (sizeof(double) * JF_COUNT + sizeof(int) + kRecMax) +
           (size_t)stage_cap_ * (sizeof(double) * JF_COUNT + 2 * sizeof(int));
}

int Engine::prepare_batch_item(int nj, int ni, const double (*xi)[3], ForceParams &item, cudaEvent_t ready,
                               unsigned *status, void *dst) {
    if (!open_ && open(env_int("G6B200_DEVICE", 0), 0)) return -1;
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    const int km = kmode();
    const int T = tile_size(km);
    const int nj_pad = round_up(nj, T);
    if (nj_pad > 0 && ensure_capacity(nj_pad - 1)) return -1;
    double xm = xmax_;
    for (int i = 0; i < ni; ++i)
        for (int c = 0; c < 3; ++c) xm = std::max(xm, std::fabs(xi[i][c]));
    xmax_ = xm;
    if (flush_j()) return -1;
    const int E = std::max(E_, choose_E(xmax_));
    if (E != E_) {
        E_ = E;
        pred_valid_ = false;
    }
    const FixedScale fs = scale();
    if (dst) {
        launch_predict(stream_, km, d_jraw_, d_jindex_, cap_, nj, nj_pad, ti_, fs, dst, status);
        G6_CHECK(cudaGetLastError(), "predict launch");
        stats_.launches++;
    } else if (!pred_valid_ || pred_ti_ != ti_ || pred_nj_ != nj || pred_mode_ != km || pred_E_ != E_) {
        // a range report of this prediction lands in the batch's status word
        launch_predict(stream_, km, d_jraw_, d_jindex_, cap_, nj, nj_pad, ti_, fs, d_jrec_, status);
        G6_CHECK(cudaGetLastError(), "predict launch");
        stats_.launches++;
        pred_valid_ = true;
        pred_ti_ = ti_;
        pred_nj_ = nj;
        pred_mode_ = km;
        pred_E_ = E_;
    }
    G6_CHECK(cudaEventRecord(ready, stream_), "event");
    item.jrec = dst ? dst : d_jrec_;
    item.nj = nj;
    item.nj_pad = nj_pad;
    item.fs = fs;
    stats_.calls++;
    stats_.interactions += (long long)ni * nj;
    return 0;
}

int Engine::read_neighbours() {
    if (!open_) return -1;
    if (!call_nb_) {
        nb_host_.clear();
        nb_read_ = true;
        return 0;
    }
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    G6_CHECK(cudaEventSynchronize(ev_done_), "wait");
    const long long total = h_nb_off_[call_ni_];
    nb_host_.resize((size_t)total);
    if (total > 0) {
        G6_CHECK(cudaMemcpy(nb_host_.data(), d_nb_sorted_, sizeof(int) * (size_t)total, cudaMemcpyDeviceToHost),
                 "nb copy");
        stats_.d2h_bytes += 4 * total;
    }
    nb_read_ = true;
    for (int i = 0; i < call_ni_; ++i)
        if (h_nb_count_[i] > nb_cap_) return 1;
    return 0;
}

int Engine::neighbour_count(int pipe) const {
    if (!nb_read_ || pipe < 0 || pipe >= call_ni_) return -1;
    return call_nb_ ? h_nb_count_[pipe] : 0;
}

int Engine::neighbours_all(int pipe, int *nbl) {
    const int count = neighbour_count(pipe);
    if (count <= 0) return count;
    if (count <= nb_cap_) {
        memcpy(nbl, nb_host_.data() + h_nb_off_[pipe], sizeof(int) * count);
        return count;
    }
    if (!call_g4_ || kmode() != kKernF64) {
        last_error = "g6b200: full neighbour lists need a GRAPE-4 call";
        return -1;
    }
    // Longer than the force kernel's per-i capacity: one pass over the
    // predicted j-set (still in d_jrec_) for this pipe alone.
    G6_CHECK(cudaSetDevice(device_), "cudaSetDevice");
    int *d_buf = nullptr;
    G6_CHECK(cudaMalloc(&d_buf, sizeof(int) * ((size_t)count + 1)), "nb full");
    cudaError_t e = launch_nb_full_g4(stream_, d_jrec_, call_nj_, h_irec_[pipe], h_ieps2_[pipe], d_buf + 1, count,
                                      d_buf);
    int got = -1;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&got, d_buf, sizeof(int), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nbl, d_buf + 1, sizeof(int) * count, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    cudaFree(d_buf);
    if (e != cudaSuccess) return fail("nb full", e);
    stats_.launches++;
    stats_.d2h_bytes += 4LL * (count + 1);
    if (got != count) {
        last_error = "g6b200: full neighbour pass disagrees with the force kernel's count";
        return -1;
    }
    return count;
}

int Engine::get_neighbours(int pipe, int max_length, int *nblen, int *nbl) {
    if (!nb_read_ || pipe < 0 || pipe >= call_ni_) {
        if (nblen) *nblen = 0;
        return -1;
    }
    if (!call_nb_) {
        *nblen = 0;
        return 0;
    }
    const int count = h_nb_count_[pipe];
    const long long off = h_nb_off_[pipe];
    const int stored = (int)(h_nb_off_[pipe + 1] - off);
    if (count > max_length || count > nb_cap_) {
        const int n = std::min(max_length, stored);
        if (n > 0) memcpy(nbl, nb_host_.data() + off, sizeof(int) * n);
        *nblen = max_length;
        return 1;
    }
    if (stored > 0) memcpy(nbl, nb_host_.data() + off, sizeof(int) * stored);
    *nblen = stored;
    return 0;
}

}  // namespace g6
