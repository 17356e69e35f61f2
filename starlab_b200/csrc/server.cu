// server.cu -- continuous batching of force calls from many clusters.
//
// Clients (host threads, e.g. kira-like integrations each owning one
// cluster) submit force calls -- a block time, an i-block and its predicted
// positions/velocities, exactly the content of one g6calc_firsthalf_ -- and
// later wait for the results (g6calc_lasthalf2_'s outputs).  A dispatcher
// thread takes every pending call of its lane, prepares each call's j-set
// (the cluster's staged updates, then a prediction to the call's block time
// into a buffer of the call's own, so two calls of one cluster may share a
// batch) on that cluster's stream, and runs all calls as ONE launch over
// their (call, i-tile, j-split) work list.  A call sees the j-particles
// loaded before its batch is dispatched.  Calls that arrive while a batch is
// on the GPU join the next one.  Each call's split plan depends on its own
// sizes only, so its results are bit-identical alone and in any mix.
//
// Cluster j-state stays resident on the device.  Admission: opening a
// cluster reserves its HBM footprint against a budget; when the budget is
// exhausted the opener waits until another cluster is closed.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "engine.h"
#include "kernels.h"

namespace g6 {

void record_error(const std::string &msg);

struct Request {
    long long id;
    int cluster;
    int lane;
    double ti, eps2;
    int nj, ni;
    std::vector<int> index;
    std::vector<double> xi, vi;  // [ni][3]
    // results
    std::vector<double> acc, jerk, pot;
    std::vector<int> nn;
    int rc = 0;
    bool done = false;
    double t_submit = 0, t_done = 0;
    long long batch = -1;  // sequence number of the batch that ran the call
    int batch_size = 0;    // calls in that batch
    std::condition_variable cv;  // signalled once, when done (waits on the server mutex)
};

// Per-batch and per-call timing records, kept when G6B200_SRV_TRACE names a
// file (written as CSV at shutdown): where the time of a served call goes.
struct BatchTrace {
    int lane, nb;
    long long ni_total, interactions;
    double t_begin, t_launch, t_end, gpu_ms;
    int grew;
};
struct CallTrace {
    long long id;
    int lane, cluster, ni, nj;
    double t_submit, t_batch, t_done;
};

struct ServerStats {
    long long batches = 0, requests = 0, interactions = 0, max_batch = 0;
    double gpu_ms = 0;      // device time of the batches (events)
    double batch_ms = 0;    // host wall time inside run_batch
    double queue_ms = 0;    // summed time calls waited before their batch started
};

class Server;

// One dispatch lane: its own stream (with a priority), buffers and thread.
// Lane 0 takes small calls and launches persistently on a high-priority
// stream; lane 1 takes large calls, one CTA per task on a low-priority
// stream, so small-call CTAs are scheduled as large-call CTAs retire.
struct Lane {
    int id = 0;
    bool persistent = true;
    std::deque<std::shared_ptr<Request>> pending;
    std::thread thread;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_clear = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    std::vector<cudaEvent_t> ready;  // one per call slot
    size_t cap_i = 0, cap_part = 0, cap_jrec = 0;
    int cap_items = 0;
    IRec *h_irec = nullptr, *d_irec = nullptr;
    unsigned char *h_out = nullptr, *d_out = nullptr;
    Partial *d_part = nullptr;
    unsigned char *d_jrec = nullptr;
    ForceParams *h_items = nullptr, *d_items = nullptr;
    int *h_pre = nullptr, *d_pre = nullptr;
    int *d_counter = nullptr;
    int *d_tcnt = nullptr;  // [cap_i] i-tile arrival counters, zero between batches
    std::vector<void *> retired_host;  // pinned buffers replaced by larger ones (freed at shutdown)
};

class Server {
  public:
    Server(int device, long long budget, int precision, int max_batch)
        : device_(device), budget_(budget), precision_(precision), max_batch_(max_batch > 0 ? max_batch : 1024) {}
    ~Server() { shutdown(); }

    std::string err;

    int start();
    void shutdown();
    int open_cluster(long long n_cap, double eps2);  // blocks until admitted
    int close_cluster(int c);
    int set_j(int c, int n, const int *address, const double *tj, const double *mass, const double (*j6)[3],
              const double (*a2)[3], const double (*v)[3], const double (*x)[3]);
    long long submit(int c, double ti, int nj, int ni, const int *index, const double (*xi)[3],
                     const double (*vi)[3]);
    int wait(long long id, double (*acc)[3], double (*jerk)[3], double *pot, int *nn, double *latency_s,
             long long *batch = nullptr, int *batch_size = nullptr);
    // While held, no lane takes new calls; on release every pending call of
    // a lane (up to max_batch) goes into its next batch together.
    void hold(bool on) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            held_ = on;
        }
        cv_work_.notify_all();
    }
    ServerStats stats() {
        std::lock_guard<std::mutex> lk(mu_);
        return stats_;
    }

  private:
    struct Cluster {
        std::unique_ptr<Engine> eng;
        std::mutex mu;
        long long footprint = 0;
        double eps2 = 0;
        int inflight = 0;  // calls pending or running
    };
    void loop(Lane &L);
    int run_batch(Lane &L, std::vector<std::shared_ptr<Request>> &batch);
    int ensure(Lane &L, size_t ni_total, size_t parts, size_t jrec_bytes, int n_items);
    void free_lane(Lane &L);
    static double now() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }

    int device_;
    long long budget_, used_ = 0;
    int precision_, max_batch_;
    int kmode_ = kKernMixedP;
    long long small_max_ = 100000000;  // calls with ni * nj <= this go to lane 0
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_, cv_mem_;
    std::map<int, std::unique_ptr<Cluster>> clusters_;
    int next_cluster_ = 0;
    std::map<long long, std::shared_ptr<Request>> inflight_;
    long long next_id_ = 1;
    bool stop_ = false;
    bool held_ = false;
    long long batch_seq_ = 0;
    bool started_ = false;
    ServerStats stats_;
    std::string trace_path_;
    double t_created_ = now();
    std::vector<BatchTrace> batch_trace_;
    std::vector<CallTrace> call_trace_;
    void write_trace();
    Lane lanes_[2];
    int ctas_ = 0;
    ForceConfig cfg_{};
};

int Server::start() {
    if (cudaSetDevice(device_) != cudaSuccess) {
        err = "server: bad device";
        return -1;
    }
    if (const char *e = getenv("G6B200_SRV_SMALL")) small_max_ = atoll(e);
    if (const char *e = getenv("G6B200_SRV_TRACE")) trace_path_ = e;
    kmode_ = precision_ == kModeF64 ? kKernF64 : kKernMixedP;
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);  // hi = greatest priority (numerically lowest)
    for (int k = 0; k < 2; ++k) {
        Lane &L = lanes_[k];
        L.id = k;
        L.persistent = k == 0;
        if (cudaStreamCreateWithPriority(&L.stream, cudaStreamNonBlocking, k == 0 ? hi : lo) != cudaSuccess ||
            cudaEventCreateWithFlags(&L.ev_clear, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&L.ev_t0) != cudaSuccess || cudaEventCreate(&L.ev_t1) != cudaSuccess ||
            cudaMalloc(&L.d_counter, 16) != cudaSuccess) {
            err = "server: CUDA setup failed";
            return -1;
        }
    }
    cfg_ = batch_config(kmode_);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
    ctas_ = batch_ctas(kmode_, cfg_, sms);
    // Pre-size the lanes (i-records, split partials, per-call predicted
    // j-sets, work items) for batches of tens of clusters of up to 2^17
    // particles: about 0.4 GB of HBM and 50 MB of pinned host memory.
    const size_t rec = kmode_ == kKernF64 ? sizeof(JRecF64) : sizeof(JRecMixed);
    if (ensure(lanes_[0], 1 << 17, 1 << 19, rec << 21, 1024) || ensure(lanes_[1], 1 << 18, 1 << 19, rec << 22, 256) ||
        cudaStreamSynchronize(lanes_[0].stream) != cudaSuccess || cudaStreamSynchronize(lanes_[1].stream) != cudaSuccess) {
        err = "server: lane buffers";
        return -1;
    }
    for (int k = 0; k < 2; ++k) lanes_[k].thread = std::thread([this, k] { loop(lanes_[k]); });
    started_ = true;
    return 0;
}

void Server::free_lane(Lane &L) {
    if (L.stream) cudaStreamSynchronize(L.stream);
    for (void *p : L.retired_host) cudaFreeHost(p);
    if (L.h_irec) cudaFreeHost(L.h_irec);
    if (L.h_out) cudaFreeHost(L.h_out);
    if (L.h_items) cudaFreeHost(L.h_items);
    if (L.h_pre) cudaFreeHost(L.h_pre);
    for (void *p : {(void *)L.d_irec, (void *)L.d_out, (void *)L.d_part, (void *)L.d_items, (void *)L.d_pre,
                    (void *)L.d_jrec, (void *)L.d_tcnt})
        if (p) cudaFreeAsync(p, L.stream);
    if (L.d_counter) cudaFree(L.d_counter);
    if (L.stream) cudaStreamSynchronize(L.stream);
    for (cudaEvent_t e : L.ready) cudaEventDestroy(e);
    L.ready.clear();
    for (cudaEvent_t e : {L.ev_clear, L.ev_t0, L.ev_t1})
        if (e) cudaEventDestroy(e);
    if (L.stream) cudaStreamDestroy(L.stream);
    L = Lane();
}

void Server::shutdown() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (stop_) return;
        stop_ = true;
    }
    cv_work_.notify_all();
    cv_mem_.notify_all();
    for (Lane &L : lanes_)
        if (L.thread.joinable()) L.thread.join();
    write_trace();
    cudaSetDevice(device_);
    for (auto &kv : clusters_) kv.second->eng.reset();
    clusters_.clear();
    for (Lane &L : lanes_) free_lane(L);
}

int Server::open_cluster(long long n_cap, double eps2) {
    // footprint: raw j-state + records + staging, as Engine allocates it
    const long long foot = ((n_cap + 255) / 256 * 256) * (8LL * JF_COUNT + 4 + 64) + 16384LL * (8 * JF_COUNT + 8);
    std::unique_lock<std::mutex> lk(mu_);
    if (foot > budget_) {
        err = "server: cluster larger than the whole HBM budget";
        return -1;
    }
    cv_mem_.wait(lk, [&] { return stop_ || used_ + foot <= budget_; });
    if (stop_) return -1;
    used_ += foot;
    const int id = next_cluster_++;
    auto cl = std::make_unique<Cluster>();
    cl->footprint = foot;
    cl->eps2 = eps2;
    cl->eng = std::make_unique<Engine>(200000 + id);
    lk.unlock();
    Engine &e = *cl->eng;
    if (e.open(device_, (int)n_cap) || e.set_mode(precision_) || e.set_npipes((int)std::max<long long>(n_cap, 1))) {
        err = "server: " + e.last_error;
        lk.lock();
        used_ -= foot;
        cv_mem_.notify_all();
        return -1;
    }
    lk.lock();
    clusters_[id] = std::move(cl);
    return id;
}

int Server::close_cluster(int c) {
    std::unique_ptr<Cluster> cl;
    {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = clusters_.find(c);
        if (it == clusters_.end()) return -1;
        Cluster *p = it->second.get();
        cv_done_.wait(lk, [&] { return p->inflight == 0; });
        cl = std::move(it->second);
        clusters_.erase(it);
        used_ -= cl->footprint;
    }
    cv_mem_.notify_all();
    cl->eng.reset();
    return 0;
}

int Server::set_j(int c, int n, const int *address, const double *tj, const double *mass, const double (*j6)[3],
                  const double (*a2)[3], const double (*v)[3], const double (*x)[3]) {
    Cluster *cl;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = clusters_.find(c);
        if (it == clusters_.end()) return -1;
        cl = it->second.get();
    }
    std::lock_guard<std::mutex> lk(cl->mu);
    if (cl->eng->set_j_bulk(n, address, address, tj, mass, nullptr, &j6[0][0], &a2[0][0], &v[0][0], &x[0][0])) {
        err = cl->eng->last_error;
        return -1;
    }
    return 0;
}

long long Server::submit(int c, double ti, int nj, int ni, const int *index, const double (*xi)[3],
                         const double (*vi)[3]) {
    if (ni < 0 || nj <= 0 || (ni > 0 && (!index || !xi || !vi))) return -1;  // before copying the arrays
    auto r = std::make_shared<Request>();
    r->cluster = c;
    r->ti = ti;
    r->nj = nj;
    r->ni = ni;
    r->index.assign(index, index + ni);
    r->xi.assign(&xi[0][0], &xi[0][0] + 3 * (size_t)ni);
    r->vi.assign(&vi[0][0], &vi[0][0] + 3 * (size_t)ni);
    r->lane = (long long)ni * nj <= small_max_ ? 0 : 1;
    r->t_submit = now();
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = clusters_.find(c);
        if (it == clusters_.end() || ni < 0 || nj <= 0 || stop_) return -1;
        r->eps2 = it->second->eps2;
        it->second->inflight++;
        r->id = next_id_++;
        lanes_[r->lane].pending.push_back(r);
        inflight_[r->id] = r;
    }
    cv_work_.notify_all();
    return r->id;
}

int Server::wait(long long id, double (*acc)[3], double (*jerk)[3], double *pot, int *nn, double *latency_s,
                 long long *batch, int *batch_size) {
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = inflight_.find(id);
        if (it == inflight_.end()) return -1;
        r = it->second;
        r->cv.wait(lk, [&] { return r->done; });
        inflight_.erase(id);
    }
    if (r->rc) return r->rc;
    const size_t n = r->ni;
    if (acc) memcpy(acc, r->acc.data(), 24 * n);
    if (jerk) memcpy(jerk, r->jerk.data(), 24 * n);
    if (pot) memcpy(pot, r->pot.data(), 8 * n);
    if (nn) memcpy(nn, r->nn.data(), 4 * n);
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    if (batch) *batch = r->batch;
    if (batch_size) *batch_size = r->batch_size;
    return 0;
}

void Server::loop(Lane &L) {
    cudaSetDevice(device_);
    for (;;) {
        std::vector<std::shared_ptr<Request>> batch;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_work_.wait(lk, [&] { return stop_ || (!held_ && !L.pending.empty()); });
            if (stop_ && L.pending.empty()) return;
            while (!L.pending.empty() && (int)batch.size() < max_batch_) {
                batch.push_back(L.pending.front());
                L.pending.pop_front();
            }
            const long long seq = batch_seq_++;
            for (auto &r : batch) {
                r->batch = seq;
                r->batch_size = (int)batch.size();
            }
        }
        const double tb0 = now();
        int rc = run_batch(L, batch);
        const double t = now();
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (auto &r : batch) {
                if (rc) r->rc = rc;
                r->done = true;
                r->t_done = t;
                if (!trace_path_.empty())
                    call_trace_.push_back({r->id, L.id, r->cluster, r->ni, r->nj, r->t_submit - t_created_,
                                           tb0 - t_created_, t - t_created_});
                stats_.queue_ms += (tb0 - r->t_submit) * 1e3;
                auto it = clusters_.find(r->cluster);
                if (it != clusters_.end()) it->second->inflight--;
                r->cv.notify_all();
            }
            stats_.batch_ms += (t - tb0) * 1e3;
        }
        cv_done_.notify_all();  // close_cluster waiters
    }
}

// Lane buffers grow geometrically.  Growth never synchronises the device
// (the other lane keeps running): device buffers are stream-ordered
// allocations on the lane's own stream, and replaced pinned buffers are kept
// until shutdown instead of being freed (cudaFreeHost may synchronise).
// start() pre-sizes both lanes so that growth is rare in service.
int Server::ensure(Lane &L, size_t ni_total, size_t parts, size_t jrec_bytes, int n_items) {
    auto dev_realloc = [&](auto *&ptr, size_t bytes) {
        if (ptr) cudaFreeAsync(ptr, L.stream);
        ptr = nullptr;
        return cudaMallocAsync(reinterpret_cast<void **>(&ptr), bytes, L.stream) == cudaSuccess;
    };
    auto host_realloc = [&](auto *&ptr, size_t bytes) {
        if (ptr) L.retired_host.push_back(ptr);
        ptr = nullptr;
        return cudaMallocHost(reinterpret_cast<void **>(&ptr), bytes) == cudaSuccess;
    };
    if (ni_total > L.cap_i) {
        size_t n = std::max(ni_total, L.cap_i * 2);
        if (!host_realloc(L.h_irec, sizeof(IRec) * n) || !dev_realloc(L.d_irec, sizeof(IRec) * n) ||
            !host_realloc(L.h_out, 16 + 60 * n) || !dev_realloc(L.d_out, 16 + 60 * n) ||
            !dev_realloc(L.d_tcnt, sizeof(int) * n) ||
            cudaMemsetAsync(L.d_tcnt, 0, sizeof(int) * n, L.stream) != cudaSuccess)
            return -1;
        L.cap_i = n;
    }
    if (parts > L.cap_part) {
        size_t n = std::max(parts, L.cap_part * 2);
        if (!dev_realloc(L.d_part, sizeof(Partial) * n)) return -1;
        L.cap_part = n;
    }
    if (jrec_bytes > L.cap_jrec) {
        size_t n = std::max(jrec_bytes, L.cap_jrec * 2);
        if (!dev_realloc(L.d_jrec, n)) return -1;
        L.cap_jrec = n;
    }
    if (n_items > L.cap_items) {
        int n = std::max(n_items, L.cap_items * 2);
        if (!host_realloc(L.h_items, sizeof(ForceParams) * n) || !dev_realloc(L.d_items, sizeof(ForceParams) * n) ||
            !host_realloc(L.h_pre, sizeof(int) * 2 * (n + 1)) || !dev_realloc(L.d_pre, sizeof(int) * 2 * (n + 1)))
            return -1;
        L.cap_items = n;
    }
    while ((int)L.ready.size() < n_items) {
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming)) return -1;
        L.ready.push_back(e);
    }
    return 0;
}

int Server::run_batch(Lane &L, std::vector<std::shared_ptr<Request>> &batch) {
    const int nb = (int)batch.size();
    if (nb == 0) return 0;
    const double t_begin = now();
    const size_t caps_before = L.cap_i + L.cap_part + L.cap_jrec + (size_t)L.cap_items;
    const int T = tile_of(kmode_);
    const size_t rec = kmode_ == kKernF64 ? sizeof(JRecF64) : sizeof(JRecMixed);
    size_t ni_total = 0, parts = 0, jbytes = 0;
    // Split partials by each call's own plan (batch_plan depends on the
    // call's ni and nj only), so that large i-blocks -- one split -- need none.
    auto split_of = [&](const Request &r) {
        ForceParams q{};
        q.ni = r.ni;
        q.nj_pad = (r.nj + T - 1) / T * T;
        int nt = 0;
        batch_plan(kmode_, cfg_, q, nt);
        return q.nsplit > 1 ? (size_t)q.nsplit : 0;
    };
    for (auto &r : batch) {
        const int nj_pad = (r->nj + T - 1) / T * T;
        ni_total += r->ni;
        parts += (size_t)r->ni * split_of(*r);
        jbytes += (size_t)nj_pad * rec;
    }
    if (ensure(L, std::max<size_t>(ni_total, 1), std::max<size_t>(parts, 1), std::max<size_t>(jbytes, 256), nb))
        return -3;
    unsigned *d_status = reinterpret_cast<unsigned *>(L.d_out);
    cudaMemsetAsync(L.d_out, 0, 16, L.stream);
    cudaEventRecord(L.ev_clear, L.stream);
    size_t ioff = 0, poff = 0, joff = 0;
    int task = 0;
    bool ident = true;
    double *oacc = reinterpret_cast<double *>(L.d_out + 16);
    double *ojerk = oacc + 3 * ni_total;
    double *opot = ojerk + 3 * ni_total;
    int *onn = reinterpret_cast<int *>(opot + ni_total);
    for (int k = 0; k < nb; ++k) {
        Request &r = *batch[k];
        Cluster *cl;
        {
            std::lock_guard<std::mutex> lk(mu_);
            cl = clusters_[r.cluster].get();
        }
        ForceParams p{};
        const int nj_pad = (r.nj + T - 1) / T * T;
        {
            std::lock_guard<std::mutex> lk(cl->mu);
            cl->eng->wait_event(L.ev_clear);
            cl->eng->set_ti(r.ti);
            if (cl->eng->prepare_batch_item(r.nj, r.ni, reinterpret_cast<const double(*)[3]>(r.xi.data()), p,
                                            L.ready[k], d_status, L.d_jrec + joff))
                return -2;
            ident &= cl->eng->identity_index();
        }
        cudaStreamWaitEvent(L.stream, L.ready[k], 0);
        for (int i = 0; i < r.ni; ++i) {
            IRec &q = L.h_irec[ioff + i];
            for (int c = 0; c < 3; ++c) {
                q.x[c] = r.xi[3 * i + c];
                q.v[c] = r.vi[3 * i + c];
            }
            q.h2 = 0;
            q.index = r.index[i];
            q.pad = 0;
        }
        p.irec = L.d_irec + ioff;
        p.ni = r.ni;
        p.eps2 = r.eps2;
        p.part = L.d_part + poff;
        p.out_acc = oacc + 3 * ioff;
        p.out_jerk = ojerk + 3 * ioff;
        p.out_pot = opot + ioff;
        p.out_nn = onn + ioff;
        p.status = d_status;
        p.tile_counter = L.d_tcnt + ioff;  // the last CTA of an i-tile adds its splits
        int nt = 0;
        batch_plan(kmode_, cfg_, p, nt);
        L.h_items[k] = p;
        L.h_pre[k] = task;
        L.h_pre[nb + 1 + k] = (int)ioff;
        task += nt;
        ioff += r.ni;
        poff += (size_t)r.ni * (p.nsplit > 1 ? (size_t)p.nsplit : 0);
        joff += (size_t)nj_pad * rec;
    }
    L.h_pre[nb] = task;
    L.h_pre[2 * nb + 1] = (int)ioff;
    const double t_launch = now();
    cudaEventRecord(L.ev_t0, L.stream);
    cudaMemcpyAsync(L.d_irec, L.h_irec, sizeof(IRec) * ni_total, cudaMemcpyHostToDevice, L.stream);
    cudaMemcpyAsync(L.d_items, L.h_items, sizeof(ForceParams) * nb, cudaMemcpyHostToDevice, L.stream);
    cudaMemcpyAsync(L.d_pre, L.h_pre, sizeof(int) * 2 * (nb + 1), cudaMemcpyHostToDevice, L.stream);
    if (L.persistent) cudaMemsetAsync(L.d_counter, 0, sizeof(int), L.stream);
    BatchArgs a;
    a.items = L.d_items;
    a.task0 = L.d_pre;
    a.ipre = L.d_pre + nb + 1;
    a.n_items = nb;
    a.H = cfg_.H;
    a.counter = L.d_counter;
    a.one_task_per_cta = L.persistent ? 0 : 1;
    cudaError_t e = cudaSuccess;
    if (task > 0)
        e = launch_force_batch(L.stream, kmode_, cfg_, a, L.persistent ? ctas_ : task, 0, false, ident);
    if (e != cudaSuccess) return -3;
    cudaMemcpyAsync(L.h_out, L.d_out, 16 + 60 * ni_total, cudaMemcpyDeviceToHost, L.stream);
    cudaEventRecord(L.ev_t1, L.stream);
    if (cudaStreamSynchronize(L.stream) != cudaSuccess) return -3;
    float ms = 0;
    cudaEventElapsedTime(&ms, L.ev_t0, L.ev_t1);
    const unsigned status = *reinterpret_cast<unsigned *>(L.h_out);
    if (status & ST_TMA_TIMEOUT) {  // results invalid; a task may have left its counter raised
        cudaMemsetAsync(L.d_tcnt, 0, sizeof(int) * L.cap_i, L.stream);
        cudaStreamSynchronize(L.stream);
        err = "server: j-tile copy wait timed out on the device";
        return -5;
    }
    long long inter = 0;
    if (status & ST_RANGE) {
        // rare: redo each call alone with a widened fixed-point range
        for (auto &rp : batch) {
            Request &r = *rp;
            Cluster *cl;
            {
                std::lock_guard<std::mutex> lk(mu_);
                cl = clusters_[r.cluster].get();
            }
            std::lock_guard<std::mutex> lk(cl->mu);
            Engine &eng = *cl->eng;
            eng.widen_range();
            eng.set_ti(r.ti);
            r.acc.resize(3 * (size_t)r.ni);
            r.jerk.resize(3 * (size_t)r.ni);
            r.pot.resize(r.ni);
            r.nn.resize(r.ni);
            if (eng.firsthalf(r.nj, r.ni, r.index.data(), reinterpret_cast<const double(*)[3]>(r.xi.data()),
                              reinterpret_cast<const double(*)[3]>(r.vi.data()), r.eps2, nullptr) ||
                eng.lasthalf(r.ni, reinterpret_cast<double(*)[3]>(r.acc.data()),
                             reinterpret_cast<double(*)[3]>(r.jerk.data()), r.pot.data(), r.nn.data()))
                r.rc = -4;
            inter += (long long)r.ni * r.nj;
        }
    } else {
        const unsigned char *base = L.h_out + 16;
        const double *hacc = reinterpret_cast<const double *>(base);
        const double *hjerk = hacc + 3 * ni_total;
        const double *hpot = hjerk + 3 * ni_total;
        const int *hnn = reinterpret_cast<const int *>(hpot + ni_total);
        size_t o = 0;
        for (auto &rp : batch) {
            Request &r = *rp;
            r.acc.assign(hacc + 3 * o, hacc + 3 * (o + r.ni));
            r.jerk.assign(hjerk + 3 * o, hjerk + 3 * (o + r.ni));
            r.pot.assign(hpot + o, hpot + o + r.ni);
            r.nn.assign(hnn + o, hnn + o + r.ni);
            o += r.ni;
            inter += (long long)r.ni * r.nj;
        }
    }
    {
        std::lock_guard<std::mutex> lk(mu_);
        stats_.batches++;
        stats_.requests += nb;
        stats_.interactions += inter;
        stats_.max_batch = std::max<long long>(stats_.max_batch, nb);
        stats_.gpu_ms += ms;
        if (!trace_path_.empty()) {
            const size_t caps_after = L.cap_i + L.cap_part + L.cap_jrec + (size_t)L.cap_items;
            batch_trace_.push_back({L.id, nb, (long long)ni_total, inter, t_begin - t_created_,
                                    t_launch - t_created_, now() - t_created_, ms, caps_after != caps_before});
        }
    }
    return 0;
}

void Server::write_trace() {
    if (trace_path_.empty()) return;
    FILE *f = fopen(trace_path_.c_str(), "w");
    if (!f) return;
    fprintf(f, "kind,lane,n,ni,interactions_or_nj,t0,t1,t2,gpu_ms_or_cluster,grew_or_id\n");
    for (const BatchTrace &b : batch_trace_)
        fprintf(f, "batch,%d,%d,%lld,%lld,%.6f,%.6f,%.6f,%.4f,%d\n", b.lane, b.nb, b.ni_total, b.interactions,
                b.t_begin, b.t_launch, b.t_end, b.gpu_ms, b.grew);
    for (const CallTrace &c : call_trace_)
        fprintf(f, "call,%d,1,%d,%d,%.6f,%.6f,%.6f,%d,%lld\n", c.lane, c.ni, c.nj, c.t_submit, c.t_batch, c.t_done,
                c.cluster, c.id);
    fclose(f);
}

}  // namespace g6

// ---------------------------------------------------------------------------
#pragma GCC visibility push(default)
#include "../../include/g6b200.h"
#pragma GCC visibility pop

struct g6b200_server {
    g6::Server *s;
};

extern "C" {

__attribute__((visibility("default"))) g6b200_server *g6b200_srv_create(int device, long long hbm_budget_bytes,
                                                                       int precision, int max_batch) {
    auto *s = new g6::Server(device, hbm_budget_bytes, precision, max_batch);
    if (s->start()) {
        g6::record_error(s->err);
        delete s;
        return nullptr;
    }
    return new g6b200_server{s};
}

__attribute__((visibility("default"))) int g6b200_srv_open_cluster(g6b200_server *h, long long n_cap,
                                                                   double eps2) {
    int rc = h->s->open_cluster(n_cap, eps2);
    if (rc < 0) g6::record_error(h->s->err);
    return rc;
}

__attribute__((visibility("default"))) int g6b200_srv_close_cluster(g6b200_server *h, int cluster) {
    return h->s->close_cluster(cluster);
}

__attribute__((visibility("default"))) int g6b200_srv_set_j(g6b200_server *h, int cluster, int n,
                                                            const int *address, const double *tj,
                                                            const double *mass, const double (*j6)[3],
                                                            const double (*a2)[3], const double (*v)[3],
                                                            const double (*x)[3]) {
    int rc = h->s->set_j(cluster, n, address, tj, mass, j6, a2, v, x);
    if (rc) g6::record_error(h->s->err);
    return rc;
}

__attribute__((visibility("default"))) long long g6b200_srv_submit(g6b200_server *h, int cluster, double ti,
                                                                   int nj, int ni, const int *index,
                                                                   const double (*xi)[3], const double (*vi)[3]) {
    return h->s->submit(cluster, ti, nj, ni, index, xi, vi);
}

__attribute__((visibility("default"))) int g6b200_srv_wait(g6b200_server *h, long long request, double (*acc)[3],
                                                           double (*jerk)[3], double *pot, int *nn,
                                                           double *latency_s) {
    return h->s->wait(request, acc, jerk, pot, nn, latency_s);
}

__attribute__((visibility("default"))) int g6b200_srv_wait_batch(g6b200_server *h, long long request,
                                                                 double (*acc)[3], double (*jerk)[3], double *pot,
                                                                 int *nn, double *latency_s, long long *batch,
                                                                 int *batch_size) {
    return h->s->wait(request, acc, jerk, pot, nn, latency_s, batch, batch_size);
}

__attribute__((visibility("default"))) void g6b200_srv_hold(g6b200_server *h, int hold) { h->s->hold(hold != 0); }

__attribute__((visibility("default"))) int g6b200_srv_stats(g6b200_server *h, g6b200_srv_stats_t *out) {
    g6::ServerStats st = h->s->stats();
    out->batches = st.batches;
    out->requests = st.requests;
    out->interactions = st.interactions;
    out->max_batch = st.max_batch;
    out->gpu_ms = st.gpu_ms;
    out->batch_ms = st.batch_ms;
    out->queue_ms = st.queue_ms;
    return 0;
}

__attribute__((visibility("default"))) void g6b200_srv_destroy(g6b200_server *h) {
    if (!h) return;
    delete h->s;
    delete h;
}

}  // extern "C"
