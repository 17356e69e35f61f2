// server.cu -- continuous batching of force calls from many clusters.
//
// Clients (host threads, e.g. kira-like integrations each owning one
// cluster) submit force calls -- a block time, an i-block and its predicted
// positions/velocities, exactly the content of one g6calc_firsthalf_ -- and
// later wait for the results (g6calc_lasthalf2_'s outputs).  A dispatcher
// thread takes every pending call (at most one per cluster at a time, since a
// cluster's calls are sequential), prepares each cluster's j-memory (staged
// updates, prediction to the call's block time) on that cluster's stream, and
// runs all calls as ONE persistent launch over their (call, i-tile, j-split)
// work list.  Calls that arrive while a batch is on the GPU join the next
// one.  Each call's split plan depends on its own sizes only, so its results
// are bit-identical alone and in any mix.
//
// Cluster j-state stays resident on the device.  Admission: opening a
// cluster reserves its HBM footprint against a budget; when the budget is
// exhausted the opener waits until another cluster is closed.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
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
};

struct ServerStats {
    long long batches = 0, requests = 0, interactions = 0, max_batch = 0;
    double gpu_ms = 0;      // device time of the batches (events)
    double batch_ms = 0;    // host wall time inside run_batch
    double queue_ms = 0;    // summed time calls waited before their batch started
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
    int wait(long long id, double (*acc)[3], double (*jerk)[3], double *pot, int *nn, double *latency_s);
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
        bool busy = false;  // a call of this cluster is in the current batch
        cudaEvent_t ready = nullptr;
    };
    void loop();
    int run_batch(std::vector<std::shared_ptr<Request>> &batch);
    int ensure(size_t ni_total, size_t parts, int n_items);
    static double now() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }

    int device_;
    long long budget_, used_ = 0;
    int precision_, max_batch_;
    int kmode_ = kKernMixedP;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_, cv_mem_;
    std::map<int, std::unique_ptr<Cluster>> clusters_;
    int next_cluster_ = 0;
    std::deque<std::shared_ptr<Request>> pending_;
    std::map<long long, std::shared_ptr<Request>> inflight_;
    long long next_id_ = 1;
    bool stop_ = false;
    std::thread thread_;
    ServerStats stats_;
    // device batch buffers
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev_clear_ = nullptr, ev_t0_ = nullptr, ev_t1_ = nullptr;
    size_t cap_i_ = 0, cap_part_ = 0;
    int cap_items_ = 0;
    IRec *h_irec_ = nullptr, *d_irec_ = nullptr;
    unsigned char *h_out_ = nullptr, *d_out_ = nullptr;  // status + per-request outputs
    Partial *d_part_ = nullptr;
    ForceParams *h_items_ = nullptr, *d_items_ = nullptr;
    int *h_pre_ = nullptr, *d_pre_ = nullptr;  // task0 [n+1] then ipre [n+1]
    int *d_counter_ = nullptr;
    int ctas_ = 0;
    ForceConfig cfg_{};
};

int Server::start() {
    if (cudaSetDevice(device_) != cudaSuccess) {
        err = "server: bad device";
        return -1;
    }
    kmode_ = precision_ == kModeF64 ? kKernF64 : kKernMixedP;
    if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_clear_, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&ev_t0_) != cudaSuccess || cudaEventCreate(&ev_t1_) != cudaSuccess ||
        cudaMalloc(&d_counter_, 16) != cudaSuccess) {
        err = "server: CUDA setup failed";
        return -1;
    }
    cfg_ = batch_config(kmode_);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
    ctas_ = batch_ctas(kmode_, cfg_, sms);
    thread_ = std::thread([this] { loop(); });
    return 0;
}

void Server::shutdown() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (stop_ && !thread_.joinable()) return;
        stop_ = true;
    }
    cv_work_.notify_all();
    if (thread_.joinable()) thread_.join();
    cudaSetDevice(device_);
    for (auto &kv : clusters_) {
        if (kv.second->ready) cudaEventDestroy(kv.second->ready);
        kv.second->eng.reset();
    }
    clusters_.clear();
    if (h_irec_) cudaFreeHost(h_irec_);
    if (h_out_) cudaFreeHost(h_out_);
    if (h_items_) cudaFreeHost(h_items_);
    if (h_pre_) cudaFreeHost(h_pre_);
    for (void *p : {(void *)d_irec_, (void *)d_out_, (void *)d_part_, (void *)d_items_, (void *)d_pre_,
                    (void *)d_counter_})
        if (p) cudaFree(p);
    h_irec_ = nullptr; h_out_ = nullptr; h_items_ = nullptr; h_pre_ = nullptr;
    d_irec_ = nullptr; d_out_ = nullptr; d_part_ = nullptr; d_items_ = nullptr; d_pre_ = nullptr;
    d_counter_ = nullptr;
    if (ev_clear_) cudaEventDestroy(ev_clear_);
    if (ev_t0_) cudaEventDestroy(ev_t0_);
    if (ev_t1_) cudaEventDestroy(ev_t1_);
    if (stream_) cudaStreamDestroy(stream_);
    ev_clear_ = ev_t0_ = ev_t1_ = nullptr;
    stream_ = nullptr;
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
    if (e.open(device_, (int)n_cap) || e.set_mode(precision_) || e.set_npipes((int)std::max<long long>(n_cap, 1)) ||
        cudaEventCreateWithFlags(&cl->ready, cudaEventDisableTiming) != cudaSuccess) {
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
        // wait until none of its calls is pending or in flight
        cv_done_.wait(lk, [&] {
            if (it->second->busy) return false;
            for (auto &r : pending_)
                if (r->cluster == c) return false;
            return true;
        });
        cl = std::move(it->second);
        clusters_.erase(it);
        used_ -= cl->footprint;
    }
    cv_mem_.notify_all();
    if (cl->ready) cudaEventDestroy(cl->ready);
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
    for (int k = 0; k < n; ++k) {
        const int a = address ? address[k] : k;
        if (cl->eng->set_j(a, a, tj[k], mass[k], nullptr, j6[k], a2[k], v[k], x[k])) {
            err = cl->eng->last_error;
            return -1;
        }
    }
    return 0;
}

long long Server::submit(int c, double ti, int nj, int ni, const int *index, const double (*xi)[3],
                         const double (*vi)[3]) {
    auto r = std::make_shared<Request>();
    r->cluster = c;
    r->ti = ti;
    r->nj = nj;
    r->ni = ni;
    r->index.assign(index, index + ni);
    r->xi.assign(&xi[0][0], &xi[0][0] + 3 * (size_t)ni);
    r->vi.assign(&vi[0][0], &vi[0][0] + 3 * (size_t)ni);
    r->t_submit = now();
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = clusters_.find(c);
        if (it == clusters_.end() || ni < 0 || nj <= 0) return -1;
        r->eps2 = it->second->eps2;
        r->id = next_id_++;
        pending_.push_back(r);
        inflight_[r->id] = r;
    }
    cv_work_.notify_one();
    return r->id;
}

int Server::wait(long long id, double (*acc)[3], double (*jerk)[3], double *pot, int *nn, double *latency_s) {
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = inflight_.find(id);
        if (it == inflight_.end()) return -1;
        r = it->second;
        cv_done_.wait(lk, [&] { return r->done; });
        inflight_.erase(id);
    }
    if (r->rc) return r->rc;
    const size_t n = r->ni;
    if (acc) memcpy(acc, r->acc.data(), 24 * n);
    if (jerk) memcpy(jerk, r->jerk.data(), 24 * n);
    if (pot) memcpy(pot, r->pot.data(), 8 * n);
    if (nn) memcpy(nn, r->nn.data(), 4 * n);
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    return 0;
}

void Server::loop() {
    cudaSetDevice(device_);
    for (;;) {
        std::vector<std::shared_ptr<Request>> batch;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_work_.wait(lk, [&] { return stop_ || !pending_.empty(); });
            if (stop_ && pending_.empty()) return;
            std::vector<std::shared_ptr<Request>> keep;
            for (auto &r : pending_) {
                Cluster *cl = clusters_.count(r->cluster) ? clusters_[r->cluster].get() : nullptr;
                if (cl && !cl->busy && (int)batch.size() < max_batch_) {
                    cl->busy = true;
                    batch.push_back(r);
                } else {
                    keep.push_back(r);
                }
            }
            pending_.assign(keep.begin(), keep.end());
        }
        const double tb0 = now();
        int rc = run_batch(batch);
        const double t = now();
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (auto &r : batch) {
                if (rc) r->rc = rc;
                r->done = true;
                r->t_done = t;
                stats_.queue_ms += (tb0 - r->t_submit) * 1e3;
                if (clusters_.count(r->cluster)) clusters_[r->cluster]->busy = false;
            }
            stats_.batch_ms += (t - tb0) * 1e3;
        }
        cv_done_.notify_all();
        cv_work_.notify_one();
    }
}

int Server::ensure(size_t ni_total, size_t parts, int n_items) {
    if (ni_total > cap_i_) {
        size_t n = std::max(ni_total, cap_i_ * 2);
        if (h_irec_) cudaFreeHost(h_irec_);
        if (d_irec_) cudaFree(d_irec_);
        if (h_out_) cudaFreeHost(h_out_);
        if (d_out_) cudaFree(d_out_);
        if (cudaMallocHost(&h_irec_, sizeof(IRec) * n) || cudaMalloc(&d_irec_, sizeof(IRec) * n) ||
            cudaMallocHost(&h_out_, 16 + 60 * n) || cudaMalloc(&d_out_, 16 + 60 * n))
            return -1;
        cap_i_ = n;
    }
    if (parts > cap_part_) {
        size_t n = std::max(parts, cap_part_ * 2);
        if (d_part_) cudaFree(d_part_);
        if (cudaMalloc(&d_part_, sizeof(Partial) * n)) return -1;
        cap_part_ = n;
    }
    if (n_items > cap_items_) {
        int n = std::max(n_items, cap_items_ * 2);
        if (h_items_) cudaFreeHost(h_items_);
        if (d_items_) cudaFree(d_items_);
        if (h_pre_) cudaFreeHost(h_pre_);
        if (d_pre_) cudaFree(d_pre_);
        if (cudaMallocHost(&h_items_, sizeof(ForceParams) * n) || cudaMalloc(&d_items_, sizeof(ForceParams) * n) ||
            cudaMallocHost(&h_pre_, sizeof(int) * 2 * (n + 1)) || cudaMalloc(&d_pre_, sizeof(int) * 2 * (n + 1)))
            return -1;
        cap_items_ = n;
    }
    return 0;
}

int Server::run_batch(std::vector<std::shared_ptr<Request>> &batch) {
    const int nb = (int)batch.size();
    if (nb == 0) return 0;
    size_t ni_total = 0, parts = 0;
    for (auto &r : batch) {
        ni_total += r->ni;
        const int nj_pad = (r->nj + tile_of(kmode_) - 1) / tile_of(kmode_) * tile_of(kmode_);
        parts += (size_t)r->ni * batch_max_split(kmode_, nj_pad);
    }
    if (ensure(std::max<size_t>(ni_total, 1), std::max<size_t>(parts, 1), nb)) return -3;
    unsigned *d_status = reinterpret_cast<unsigned *>(d_out_);
    cudaMemsetAsync(d_out_, 0, 16, stream_);
    cudaEventRecord(ev_clear_, stream_);
    // per call: i-records, item, outputs
    size_t ioff = 0, poff = 0;
    int task = 0;
    bool ident = true;
    double *oacc = reinterpret_cast<double *>(d_out_ + 16);
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
        {
            std::lock_guard<std::mutex> lk(cl->mu);
            cl->eng->wait_event(ev_clear_);
            cl->eng->set_ti(r.ti);
            if (cl->eng->prepare_batch_item(r.nj, r.ni, reinterpret_cast<const double(*)[3]>(r.xi.data()), p,
                                            cl->ready, d_status))
                return -2;
            ident &= cl->eng->identity_index();
        }
        cudaStreamWaitEvent(stream_, cl->ready, 0);
        for (int i = 0; i < r.ni; ++i) {
            IRec &q = h_irec_[ioff + i];
            for (int c = 0; c < 3; ++c) {
                q.x[c] = r.xi[3 * i + c];
                q.v[c] = r.vi[3 * i + c];
            }
            q.h2 = 0;
            q.index = r.index[i];
            q.pad = 0;
        }
        p.irec = d_irec_ + ioff;
        p.ni = r.ni;
        p.eps2 = r.eps2;
        p.part = d_part_ + poff;
        p.out_acc = oacc + 3 * ioff;
        p.out_jerk = ojerk + 3 * ioff;
        p.out_pot = opot + ioff;
        p.out_nn = onn + ioff;
        p.status = d_status;
        int nt = 0;
        batch_plan(kmode_, cfg_, p, nt);
        h_items_[k] = p;
        h_pre_[k] = task;
        h_pre_[nb + 1 + k] = (int)ioff;
        task += nt;
        ioff += r.ni;
        const int nj_pad = p.nj_pad;
        poff += (size_t)r.ni * batch_max_split(kmode_, nj_pad);
    }
    h_pre_[nb] = task;
    h_pre_[2 * nb + 1] = (int)ioff;
    cudaEventRecord(ev_t0_, stream_);
    cudaMemcpyAsync(d_irec_, h_irec_, sizeof(IRec) * ni_total, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(d_items_, h_items_, sizeof(ForceParams) * nb, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(d_pre_, h_pre_, sizeof(int) * 2 * (nb + 1), cudaMemcpyHostToDevice, stream_);
    cudaMemsetAsync(d_counter_, 0, sizeof(int), stream_);
    BatchArgs a;
    a.items = d_items_;
    a.task0 = d_pre_;
    a.ipre = d_pre_ + nb + 1;
    a.n_items = nb;
    a.H = cfg_.H;
    a.counter = d_counter_;
    cudaError_t e = launch_force_batch(stream_, kmode_, cfg_, a, ctas_, (int)ni_total, false, ident);
    if (e != cudaSuccess) return -3;
    cudaMemcpyAsync(h_out_, d_out_, 16 + 60 * ni_total, cudaMemcpyDeviceToHost, stream_);
    cudaEventRecord(ev_t1_, stream_);
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return -3;
    float ms = 0;
    cudaEventElapsedTime(&ms, ev_t0_, ev_t1_);
    const unsigned status = *reinterpret_cast<unsigned *>(h_out_);
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
        const unsigned char *base = h_out_ + 16;
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
    }
    return 0;
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
