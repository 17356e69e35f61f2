// resident.cu -- a device-resident serving loop for force calls of many
// clusters.
//
// The reference's per-call unit is force_by_grape
// (src/node/dyn/hdyn/evolve/hdyn_grape6.C:474-910): set the block time, send
// an i-block (predicted positions and velocities), read back acc, jerk, pot
// and the nearest neighbour.  Here many clients (host threads, e.g. kira-like
// integrations each owning one cluster) submit such calls, and ONE persistent
// cooperative kernel serves them with no launch per call or per batch:
//
//   host    writes a request (cluster, block time, i-records, result buffer;
//           all in pinned host memory the GPU reads and writes directly)
//           into a ring slot and marks it READY;
//   gather  CTA 0 takes every READY slot in ring order that fits the batch
//           workspace and builds each call's work item (j-record buffer,
//           i-records, outputs, split plan -- batch_plan, from the call's own
//           sizes only) and the prefix sums of tasks;
//   predict all CTAs: each call's j-set predicted to the call's block time
//           into the call's own j-record buffer; its i-records copied in;
//   force   all CTAs take (call, i-tile, j-split) tasks from one counter --
//           the process_task of the launch-per-batch kernels, so a call's
//           sums are bit-identical alone and in any mix;
//   return  all CTAs copy the results into the requests' host buffers; CTA 0
//           marks the slots DONE.
//
// Phases are separated by a grid barrier.  Every wait is bounded by the
// global timer: the ring poll ends after an idle time (the kernel exits; the
// host relaunches it when the next request comes), a grid barrier gives up
// after wait_ns (the kernel reports RES_ERR_BARRIER and exits; the host marks
// the calls it had taken failed), and the j-tile copy waits inside a task
// report ST_TMA_TIMEOUT in that call's status.  A host stop flag ends the
// loop.
//
// j-particles are kept per cluster in device memory with a pinned host
// mirror: an update writes the mirror and copies the touched rows with the
// copy engine (no kernel), so the resident kernel may hold every SM.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>
#include "force_device.cuh"
#include "kernels.h"
#include "predict_device.cuh"

namespace g6 {

void record_error(const std::string &msg);

namespace {

enum SlotState { kFree = 0, kReady = 1, kTaken = 2, kDone = 3, kFailed = 4 };
enum ResErr { RES_ERR_BARRIER = 1, RES_ERR_TOO_LARGE = 2 };
constexpr unsigned kLostWithKernel = 0x80000000u;  // slot status: the kernel left before finishing it

// One request in pinned host memory (device-visible).  The host fills the
// fields and then releases state = kReady; the device takes it (kTaken),
// writes the results and status, then releases kDone.
struct __align__(64) ResSlot {
    int state;
    int cluster;         // index into the cluster table
    int ni, nj;
    double ti, eps2;
    FixedScale fs;
    const IRec *irec;    // [ni], pinned host memory
    unsigned char *out;  // acc [ni][3], jerk [ni][3], pot [ni], nn [ni]: 60 B per i, pinned host memory
    long long batch;     // written by the device
    int batch_size;
    unsigned status;     // ST_* bits of this call
};

// Control words in pinned host memory.
struct ResCtl {
    int stop;            // host -> device: leave the loop
    int stall_once;      // host -> device: self-test, CTA 0 leaves without arriving at a barrier
    unsigned error;      // device -> host: RES_ERR_* bits
    int max_batch;       // device -> host: largest batch so far
    unsigned long long batches, calls;
};

// One cluster's raw j-state (device memory).
struct ResCluster {
    const double *jraw;  // [JF_COUNT][cap]
    const int *jindex;   // [cap]
    int cap;
    int ident;           // index == address for every j (the fast self test)
};

// What the phases need of a request, copied to device memory at gather
// (the slot itself lives in host memory).
struct ResItem {
    double ti;
    ResCluster c;
    int ni;
    const IRec *irec;    // host
    unsigned char *out;  // host
};

// Kernel parameter.
struct ResDev {
    ResSlot *slots;  // mapped ring
    int nslots;
    ResCtl *ctl;     // mapped
    const ResCluster *clusters;  // mapped
    long long *tail;  // next ring position to look at (device memory, kept across launches)
    // batch workspace (device memory)
    ForceParams *items;
    ResItem *info;
    int *task0, *ipre, *upre, *slot_of;
    int max_items;
    unsigned char *jrec;
    size_t jrec_cap;
    IRec *irec;
    double *acc, *jerk, *pot;
    int *nn;
    int *tcnt;
    size_t i_cap;
    Partial *part;
    size_t part_cap;
    unsigned *status;  // [max_items]
    int *counter;
    int *nitems;       // CTA 0 -> all: calls in this batch, -1 = leave
    int *leave;        // set by a CTA whose task failed: leave after this batch
    unsigned *bar_count, *bar_gen;
    unsigned long long idle_ns, wait_ns;
    int kmode;
    ForceConfig cfg;
};

__device__ __forceinline__ int ld_acquire_sys(const int *p) {
    int v;
    asm volatile("ld.acquire.sys.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_sys(int *p, int v) {
    asm volatile("st.release.sys.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void nap() { __nanosleep(1000); }

// Grid barrier over co-resident CTAs (cooperative launch), bounded: false
// when the other CTAs did not all arrive within limit_ns.  gen is thread 0's
// count of barriers passed.
__device__ bool grid_barrier(const ResDev &d, unsigned &gen, unsigned long long limit_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        const unsigned target = gen + 1;
        if (atomicAdd(d.bar_count, 1u) == gridDim.x - 1) {
            atomicExch(d.bar_count, 0u);
            __threadfence();
            atomicExch(d.bar_gen, target);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            while (atomicAdd(d.bar_gen, 0u) != target) {
                if (globaltimer_ns() - t0 > limit_ns) {
                    ok = 0;
                    break;
                }
                nap();
            }
        }
        gen = target;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ int find_item(const int *pre, int n, int v) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// CTA 0, one thread: take READY slots into a batch.  Returns the number of
// calls, or -1 to leave (stop flag, a failed task, or idle for idle_ns).
__device__ int gather(const ResDev &d) {
    if (atomicAdd(d.leave, 0)) return -1;
    const int T = tile_of(d.kmode);
    const size_t rec = d.kmode == kKernF64 ? sizeof(JRecF64) : sizeof(JRecMixed);
    const unsigned long long t0 = globaltimer_ns();
    long long tail = *d.tail;
    int n = 0, task = 0, units = 0;
    size_t joff = 0, ioff = 0, poff = 0;
    for (;;) {
        if (ld_acquire_sys(&d.ctl->stop)) {
            if (n == 0) return -1;
            break;
        }
        ResSlot *s = &d.slots[tail % d.nslots];
        if (n < d.max_items && ld_acquire_sys(&s->state) == kReady) {
            const int nj = s->nj, ni = s->ni;
            const int nj_pad = (nj + T - 1) / T * T;
            ForceParams p{};
            p.nj = nj;
            p.nj_pad = nj_pad;
            p.ni = ni;
            int nt = 0;
            batch_plan(d.kmode, d.cfg, p, nt);
            const size_t nparts = p.nsplit > 1 ? (size_t)ni * p.nsplit : 0;
            const int ju = d.kmode == kKernMixedP ? nj_pad / 2 : nj_pad;  // prediction units
            const bool fits = joff + (size_t)nj_pad * rec <= d.jrec_cap && ioff + ni <= d.i_cap &&
                              poff + nparts <= d.part_cap;
            if (!fits) {
                if (n > 0) break;  // the rest go into the next batch
                // larger than the whole workspace: refuse it
                s->batch = -1;
                s->status = 0;
                atomicOr(&d.ctl->error, (unsigned)RES_ERR_TOO_LARGE);
                __threadfence_system();
                st_release_sys(&s->state, kFailed);
                ++tail;
                continue;
            }
            s->state = kTaken;  // the host reads it only after kDone / kFailed
            ResItem it;
            it.ti = s->ti;
            it.c = d.clusters[s->cluster];
            it.ni = ni;
            it.irec = s->irec;
            it.out = s->out;
            p.jrec = d.jrec + joff;
            p.irec = d.irec + ioff;
            p.eps2 = s->eps2;
            p.fs = s->fs;
            p.part = d.part + poff;
            p.out_acc = d.acc + 3 * ioff;
            p.out_jerk = d.jerk + 3 * ioff;
            p.out_pot = d.pot + ioff;
            p.out_nn = d.nn + ioff;
            p.status = d.status + n;
            p.tile_counter = d.tcnt + ioff;
            d.status[n] = 0;
            d.items[n] = p;
            d.info[n] = it;
            d.slot_of[n] = (int)(tail % d.nslots);
            d.task0[n] = task;
            d.ipre[n] = (int)ioff;
            d.upre[n] = units;
            task += nt;
            units += ju + ni;
            joff += (size_t)nj_pad * rec;
            ioff += ni;
            poff += nparts;
            ++n;
            ++tail;
            continue;
        }
        if (n > 0) break;
        if (globaltimer_ns() - t0 > d.idle_ns) return -1;
        nap();
    }
    d.task0[n] = task;
    d.ipre[n] = (int)ioff;
    d.upre[n] = units;
    *d.tail = tail;
    *d.counter = 0;
    return n;
}

// One task of call k, i-lane shape IL.  Not inlined: each task body gets
// its own register allocation (inlined beside the loop's other phases, the
// shapes and self-test variants together spilled).
template <int K, bool ID, int IL>
__device__ __noinline__ bool run_task(const ForceParams *items, int k, int local, int itile, unsigned char *smem,
                                      int &gt) {
    const ForceParams p = items[k];
    const int nit = (p.ni + itile - 1) / itile;
    return process_task<K, IL, 1, false, ID, kVarUnroll4>(p, local % nit, local / nit, smem, gt);
}

template <int K, bool ID>
__device__ __forceinline__ bool run_task_any(const ForceParams *items, int k, int local, unsigned char *smem,
                                             int &gt) {
    const ForceParams &p = items[k];
    const int il = batch_il(p.ni);
    const int itile = (blockDim.x >> 5) / p.H * il;
    if (il == 32) return run_task<K, ID, 32>(items, k, local, itile, smem, gt);
    if (il == 8) return run_task<K, ID, 8>(items, k, local, itile, smem, gt);
    return run_task<K, ID, 1>(items, k, local, itile, smem, gt);
}

template <int K>
__global__ void __launch_bounds__(256, 2) resident_kernel(const ResDev d) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_task, s_n;
    init_bars(smem);
    unsigned gen = 0;
    if (threadIdx.x == 0) gen = atomicAdd(d.bar_gen, 0u);
    int gt = 0;
    bool failed = false;  // a grid barrier ran out
    for (;;) {
        // ---- gather
        if (blockIdx.x == 0) {
            if (threadIdx.x == 0) {
                *d.nitems = gather(d);
                __threadfence();
                s_n = 0;
                if (ld_acquire_sys(&d.ctl->stall_once)) {
                    // self-test of the bounded barrier: this CTA leaves without
                    // arriving, so the other CTAs' waits run out
                    st_release_sys(&d.ctl->stall_once, 0);
                    s_n = -2;
                }
            }
            __syncthreads();
            if (s_n == -2) return;
        }
        if (!grid_barrier(d, gen, d.wait_ns)) {
            failed = true;
            break;
        }
        if (threadIdx.x == 0) s_n = *(volatile int *)d.nitems;
        __syncthreads();
        const int n = s_n;
        if (n < 0) break;
        // ---- predict each call's j-set into its buffer; copy its i-records in
        const int total_units = d.upre[n];
        for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < total_units; u += gridDim.x * blockDim.x) {
            const int k = find_item(d.upre, n, u);
            const ResItem &it = d.info[k];
            const ForceParams &p = d.items[k];
            const int local = u - d.upre[k];
            const int ju = K == kKernMixedP ? p.nj_pad / 2 : p.nj_pad;
            if (local < ju) {
                if constexpr (K == kKernMixedP)
                    predict_pair_unit(it.c.jraw, it.c.jindex, it.c.cap, p.nj, local, it.ti, p.fs,
                                      reinterpret_cast<JPairMixed *>(const_cast<void *>(p.jrec)), p.status);
                else
                    predict_f64_unit(it.c.jraw, it.c.jindex, it.c.cap, p.nj, local, it.ti,
                                     reinterpret_cast<JRecF64 *>(const_cast<void *>(p.jrec)));
            } else {
                const int i = local - ju;
                const_cast<IRec *>(p.irec)[i] = it.irec[i];
            }
        }
        if (!grid_barrier(d, gen, d.wait_ns)) {
            failed = true;
            break;
        }
        // ---- force: (call, i-tile, j-split) tasks from one counter
        const int total = d.task0[n];
        for (;;) {
            __syncthreads();
            if (threadIdx.x == 0) s_task = atomicAdd(d.counter, 1);
            __syncthreads();
            const int task = s_task;
            if (task >= total) break;
            const int k = find_item(d.task0, n, task);
            const int local = task - d.task0[k];
            const bool ok = d.info[k].c.ident ? run_task_any<K, true>(d.items, k, local, smem, gt)
                                              : run_task_any<K, false>(d.items, k, local, smem, gt);
            if (!ok) {
                // a copy wait ran out (the call's status says so): this CTA
                // takes no further task, and the loop ends after this batch
                if (threadIdx.x == 0) atomicExch(d.leave, 1);
                break;
            }
        }
        if (!grid_barrier(d, gen, d.wait_ns)) {
            failed = true;
            break;
        }
        // ---- results into the requests' host buffers
        const int ni_total = d.ipre[n];
        for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ni_total; g += gridDim.x * blockDim.x) {
            const int k = find_item(d.ipre, n, g);
            const int i = g - d.ipre[k];
            const ResItem &it = d.info[k];
            const int ni = it.ni;
            double *acc = reinterpret_cast<double *>(it.out);
            double *jerk = acc + 3 * (size_t)ni;
            double *pot = jerk + 3 * (size_t)ni;
            int *nn = reinterpret_cast<int *>(pot + ni);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                acc[3 * (size_t)i + c] = d.acc[3 * (size_t)g + c];
                jerk[3 * (size_t)i + c] = d.jerk[3 * (size_t)g + c];
            }
            pot[i] = d.pot[g];
            nn[i] = d.nn[g];
        }
        __threadfence_system();
        if (!grid_barrier(d, gen, d.wait_ns)) {
            failed = true;
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long b = d.ctl->batches;
            for (int k = 0; k < n; ++k) {
                ResSlot *s = &d.slots[d.slot_of[k]];
                s->status = d.status[k];
                s->batch = (long long)b;
                s->batch_size = n;
            }
            __threadfence_system();
            for (int k = 0; k < n; ++k) st_release_sys(&d.slots[d.slot_of[k]].state, kDone);
            d.ctl->batches = b + 1;
            d.ctl->calls += n;
            if (n > d.ctl->max_batch) d.ctl->max_batch = n;
            __threadfence_system();
        }
    }
    if (failed && threadIdx.x == 0) atomicOr(&d.ctl->error, (unsigned)RES_ERR_BARRIER);
}

}  // namespace
}  // namespace g6

// ---------------------------------------------------------------------------
// Host side.

namespace g6 {

namespace {

constexpr int kResSlots = 1024;
constexpr int kResMaxItems = 1024;
constexpr int kResClusters = 4096;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// Pinned, mapped host memory for the requests' i-records and results.
// Chunks are taken with cudaHostAlloc as needed and given back only at
// shutdown: cudaFreeHost synchronises with the device, so freeing while the
// resident kernel runs would stall the caller until the kernel's idle exit.
// Inside a chunk, first fit over an offset-ordered free list, coalesced on
// release.  Called with the server's mutex held.
class PinnedArena {
  public:
    static constexpr size_t kAlign = 256;
    static constexpr size_t kChunk = 64u << 20;

    unsigned char *alloc(size_t bytes) {
        bytes = std::max(kAlign, (bytes + kAlign - 1) / kAlign * kAlign);
        for (Chunk &c : chunks_)
            for (auto it = c.free.begin(); it != c.free.end(); ++it)
                if (it->second >= bytes) {
                    const size_t off = it->first, len = it->second;
                    c.free.erase(it);
                    if (len > bytes) c.free[off + bytes] = len - bytes;
                    return c.base + off;
                }
        Chunk c;
        c.size = std::max(kChunk, (bytes + (2u << 20) - 1) / (2u << 20) * (2u << 20));
        void *q = nullptr;
        if (cudaHostAlloc(&q, c.size, cudaHostAllocMapped) != cudaSuccess) return nullptr;
        c.base = static_cast<unsigned char *>(q);
        void *dq = nullptr;
        if (cudaHostGetDevicePointer(&dq, q, 0) != cudaSuccess) {
            cudaFreeHost(q);
            return nullptr;
        }
        c.dbase = static_cast<unsigned char *>(dq);
        if (c.size > bytes) c.free[bytes] = c.size - bytes;
        chunks_.push_back(std::move(c));
        return chunks_.back().base;
    }

    void release(unsigned char *p, size_t bytes) {
        if (!p) return;
        bytes = std::max(kAlign, (bytes + kAlign - 1) / kAlign * kAlign);
        for (Chunk &c : chunks_) {
            if (p < c.base || p >= c.base + c.size) continue;
            size_t off = (size_t)(p - c.base), len = bytes;
            auto nx = c.free.lower_bound(off);
            if (nx != c.free.end() && off + len == nx->first) {
                len += nx->second;
                nx = c.free.erase(nx);
            }
            if (nx != c.free.begin()) {
                auto pv = std::prev(nx);
                if (pv->first + pv->second == off) {
                    off = pv->first;
                    len += pv->second;
                    c.free.erase(pv);
                }
            }
            c.free[off] = len;
            return;
        }
    }

    // The device's address of host address p (inside a chunk).
    unsigned char *device_ptr(unsigned char *p) const {
        for (const Chunk &c : chunks_)
            if (p >= c.base && p < c.base + c.size) return c.dbase + (p - c.base);
        return nullptr;
    }

    void destroy() {
        for (Chunk &c : chunks_) cudaFreeHost(c.base);
        chunks_.clear();
    }

  private:
    struct Chunk {
        unsigned char *base = nullptr, *dbase = nullptr;  // host and device addresses
        size_t size = 0;
        std::map<size_t, size_t> free;  // offset -> length
    };
    std::vector<Chunk> chunks_;
};

struct ResStats {
    long long batches = 0, calls = 0, launches = 0, recoveries = 0;
    int max_batch = 0;
};

class Resident {
  public:
    Resident(int device, long long budget, int precision, int max_batch)
        : device_(device), budget_(budget), precision_(precision),
          max_batch_(std::min(std::max(max_batch, 1), kResMaxItems)) {}
    ~Resident() { shutdown(); }
    std::string err;

    int start();
    void shutdown();
    int open_cluster(long long n_cap, double eps2);
    int close_cluster(int c);
    int set_j(int c, int n, const int *address, const double *tj, const double *mass, const double (*j6)[3],
              const double (*a2)[3], const double (*v)[3], const double (*x)[3]);
    long long submit(int c, double ti, int nj, int ni, const int *index, const double (*xi)[3],
                     const double (*vi)[3]);
    int wait(long long id, double (*acc)[3], double (*jerk)[3], double *pot, int *nn, double *latency_s,
             long long *batch, int *batch_size);
    void hold(bool on);
    void selftest_stall() { __atomic_store_n(&ctl_->stall_once, 1, __ATOMIC_RELEASE); }
    ResStats stats() {
        std::lock_guard<std::mutex> lk(mu_);
        ResStats s = stats_;
        s.batches = (long long)__atomic_load_n(&ctl_->batches, __ATOMIC_ACQUIRE);
        s.calls = (long long)__atomic_load_n(&ctl_->calls, __ATOMIC_ACQUIRE);
        s.max_batch = __atomic_load_n(&ctl_->max_batch, __ATOMIC_ACQUIRE);
        return s;
    }

  private:
    struct Cluster {
        long long cap = 0;
        double eps2 = 0;
        long long footprint = 0;
        double *d_raw = nullptr;  // [JF_COUNT][cap]
        int *d_index = nullptr;   // [cap]
        double *h_raw = nullptr;  // pinned mirror of d_raw
        int *h_index = nullptr;
        double xmax = 0;
        int E = -1000;
        int inflight = 0;
    };
    struct SlotHost {
        unsigned char *buf = nullptr;  // pinned, mapped (from arena_): i-records, then the results
        size_t bytes = 0;
        IRec *irec = nullptr;
        unsigned char *out = nullptr;
        double t_submit = 0;
        int cluster = -1;
        long long id = -1;
        bool held = false;
    };
    int launch_locked();
    int launch_try_locked(bool &kernel_died);
    void recover_locked();
    void fail_slots_locked(int state);
    static FixedScale scale_of(int E) {
        FixedScale fs;
        fs.to_units = std::ldexp(1.0, 23 - E);
        fs.hi_unit = std::ldexp(1.0, E - 23);
        fs.lo_unit = std::ldexp(1.0, E - 46);
        return fs;
    }

    int device_, num_sms_ = 148;
    long long budget_, used_ = 0;
    int precision_, max_batch_;
    int kmode_ = kKernMixedP;
    ForceConfig cfg_{};
    int ctas_ = 0;
    size_t smem_ = 0;
    bool started_ = false;
    cudaStream_t stream_ = nullptr, copy_ = nullptr;
    cudaEvent_t ev_run_ = nullptr;
    bool launched_ = false;
    ResSlot *slots_ = nullptr;    // pinned, mapped
    ResCtl *ctl_ = nullptr;       // pinned, mapped
    ResCluster *ctab_ = nullptr;  // pinned, mapped; one entry per cluster id
    SlotHost host_[kResSlots];
    PinnedArena arena_;
    long long head_ = 0;  // next ring position to fill
    std::vector<long long> held_;
    bool holding_ = false;
    ResDev dev_{};  // workspace pointers (device memory)
    std::vector<void *> dallocs_;
    std::mutex mu_;  // clusters, ring positions, launches
    std::condition_variable cv_mem_, cv_idle_;
    std::map<int, std::unique_ptr<Cluster>> clusters_;
    int next_cluster_ = 0;
    ResStats stats_;
};

#define RES_CHECK(call, what)                       \
    do {                                            \
        if ((call) != cudaSuccess) {                \
            err = std::string("resident: ") + what; \
            return -1;                              \
        }                                           \
    } while (0)

int Resident::start() {
    RES_CHECK(cudaSetDevice(device_), "bad device");
    kmode_ = precision_ == kModeF64 ? kKernF64 : kKernMixedP;
    cfg_ = batch_config(kmode_);
    cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, device_);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device_);
    if (!coop) {
        err = "resident: the device does not support cooperative launches";
        return -1;
    }
    const size_t tiles = 2 * (size_t)tile_of(kmode_) * jrec_bytes(kmode_);
    const size_t red = (size_t)cfg_.H * batch_itile(cfg_) * sizeof(Partial);
    smem_ = 128 + std::max(tiles, red);
    void (*fn)(const ResDev) = kmode_ == kKernF64 ? resident_kernel<kKernF64> : resident_kernel<kKernMixedP>;
    RES_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_), "smem");
    int per_sm = 0;
    RES_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem_), "occupancy");
    if (per_sm < 1) {
        err = "resident: kernel does not fit an SM";
        return -1;
    }
    ctas_ = per_sm * num_sms_;
    RES_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    RES_CHECK(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking), "stream");
    RES_CHECK(cudaEventCreateWithFlags(&ev_run_, cudaEventDisableTiming), "event");
    RES_CHECK(cudaHostAlloc(reinterpret_cast<void **>(&slots_), sizeof(ResSlot) * kResSlots, cudaHostAllocMapped),
              "ring");
    RES_CHECK(cudaHostAlloc(reinterpret_cast<void **>(&ctl_), sizeof(ResCtl), cudaHostAllocMapped), "ring");
    RES_CHECK(cudaHostAlloc(reinterpret_cast<void **>(&ctab_), sizeof(ResCluster) * kResClusters,
                            cudaHostAllocMapped), "ring");
    memset(slots_, 0, sizeof(ResSlot) * kResSlots);
    memset(ctl_, 0, sizeof(ResCtl));
    memset(ctab_, 0, sizeof(ResCluster) * kResClusters);
    ResDev &d = dev_;
    RES_CHECK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&d.slots), slots_, 0), "mapping");
    RES_CHECK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&d.ctl), ctl_, 0), "mapping");
    ResCluster *ct = nullptr;
    RES_CHECK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&ct), ctab_, 0), "mapping");
    d.clusters = ct;
    d.nslots = kResSlots;
    d.max_items = max_batch_;
    // batch workspace: j-records of 2^23 j, 2^20 i, 2^21 split partials
    const size_t rec = kmode_ == kKernF64 ? sizeof(JRecF64) : sizeof(JRecMixed);
    d.jrec_cap = rec << 23;
    d.i_cap = 1 << 20;
    d.part_cap = 1 << 21;
    auto dalloc = [&](auto *&p, size_t bytes) {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) return false;
        cudaMemset(q, 0, bytes);
        dallocs_.push_back(q);
        p = reinterpret_cast<std::remove_reference_t<decltype(p)>>(q);
        return true;
    };
    const int mi = kResMaxItems + 1;
    if (!dalloc(d.tail, 8) || !dalloc(d.items, sizeof(ForceParams) * mi) || !dalloc(d.info, sizeof(ResItem) * mi) ||
        !dalloc(d.task0, 4 * mi) || !dalloc(d.ipre, 4 * mi) || !dalloc(d.upre, 4 * mi) ||
        !dalloc(d.slot_of, 4 * mi) || !dalloc(d.jrec, d.jrec_cap) || !dalloc(d.irec, sizeof(IRec) * d.i_cap) ||
        !dalloc(d.acc, 24 * d.i_cap) || !dalloc(d.jerk, 24 * d.i_cap) || !dalloc(d.pot, 8 * d.i_cap) ||
        !dalloc(d.nn, 4 * d.i_cap) || !dalloc(d.tcnt, 4 * d.i_cap) || !dalloc(d.part, sizeof(Partial) * d.part_cap) ||
        !dalloc(d.status, 4 * mi) || !dalloc(d.counter, 4) || !dalloc(d.nitems, 4) || !dalloc(d.leave, 4) ||
        !dalloc(d.bar_count, 4) || !dalloc(d.bar_gen, 4)) {
        err = "resident: workspace allocation";
        return -1;
    }
    RES_CHECK(cudaDeviceSynchronize(), "workspace");
    const char *e = getenv("G6B200_RES_IDLE_MS");
    d.idle_ns = (unsigned long long)((e ? atof(e) : 20.0) * 1e6);
    e = getenv("G6B200_RES_WAIT_MS");
    d.wait_ns = (unsigned long long)((e ? atof(e) : 2000.0) * 1e6);
    d.kmode = kmode_;
    d.cfg = cfg_;
    started_ = true;
    return 0;
}

void Resident::shutdown() {
    if (!started_) return;
    started_ = false;
    __atomic_store_n(&ctl_->stop, 1, __ATOMIC_RELEASE);
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);  // the loop sees the stop flag within one poll
    for (void *p : dallocs_) cudaFree(p);
    dallocs_.clear();
    for (auto &kv : clusters_) {
        Cluster &c = *kv.second;
        cudaFree(c.d_raw);
        cudaFree(c.d_index);
        cudaFreeHost(c.h_raw);
        cudaFreeHost(c.h_index);
    }
    clusters_.clear();
    for (SlotHost &s : host_) s = SlotHost();
    arena_.destroy();
    cudaFreeHost(slots_);
    cudaFreeHost(ctl_);
    cudaFreeHost(ctab_);
    cudaEventDestroy(ev_run_);
    cudaStreamDestroy(stream_);
    cudaStreamDestroy(copy_);
}

int Resident::open_cluster(long long n_cap, double eps2) {
    if (n_cap < 1) n_cap = 1;
    const long long cap = (n_cap + 255) / 256 * 256;
    const long long foot = cap * (8LL * JF_COUNT + 4);
    std::unique_lock<std::mutex> lk(mu_);
    if (foot > budget_) {
        err = "resident: cluster larger than the whole HBM budget";
        return -1;
    }
    if (next_cluster_ >= kResClusters) {
        err = "resident: cluster table full";
        return -1;
    }
    cv_mem_.wait(lk, [&] { return used_ + foot <= budget_; });
    auto c = std::make_unique<Cluster>();
    c->cap = cap;
    c->eps2 = eps2;
    c->footprint = foot;
    cudaSetDevice(device_);
    if (cudaMalloc(&c->d_raw, sizeof(double) * JF_COUNT * cap) != cudaSuccess ||
        cudaMalloc(&c->d_index, sizeof(int) * cap) != cudaSuccess ||
        cudaMallocHost(&c->h_raw, sizeof(double) * JF_COUNT * cap) != cudaSuccess ||
        cudaMallocHost(&c->h_index, sizeof(int) * cap) != cudaSuccess) {
        err = "resident: cluster allocation";
        return -1;
    }
    memset(c->h_raw, 0, sizeof(double) * JF_COUNT * cap);
    for (long long j = 0; j < cap; ++j) c->h_index[j] = (int)j;
    if (cudaMemcpy(c->d_raw, c->h_raw, sizeof(double) * JF_COUNT * cap, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_index, c->h_index, sizeof(int) * cap, cudaMemcpyHostToDevice) != cudaSuccess) {
        err = "resident: cluster upload";
        return -1;
    }
    used_ += foot;
    const int id = next_cluster_++;
    ResCluster rc;
    rc.jraw = c->d_raw;
    rc.jindex = c->d_index;
    rc.cap = (int)cap;
    rc.ident = 1;
    ctab_[id] = rc;
    clusters_[id] = std::move(c);
    return id;
}

int Resident::close_cluster(int c) {
    std::unique_ptr<Cluster> cl;
    {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = clusters_.find(c);
        if (it == clusters_.end()) return -1;
        Cluster *p = it->second.get();
        cv_idle_.wait(lk, [&] { return p->inflight == 0; });
        cl = std::move(it->second);
        clusters_.erase(it);
        used_ -= cl->footprint;
    }
    cv_mem_.notify_all();
    cudaSetDevice(device_);
    cudaFree(cl->d_raw);
    cudaFree(cl->d_index);
    cudaFreeHost(cl->h_raw);
    cudaFreeHost(cl->h_index);
    return 0;
}

// j-particles go into the pinned mirror, then the touched address range of
// every row is copied to the device by the copy engine (no kernel).  Waits
// until no call of the cluster is in flight, so a running call never sees a
// half-written j-state; a call submitted after this returns sees it.
int Resident::set_j(int c, int n, const int *address, const double *tj, const double *mass, const double (*j6)[3],
                    const double (*a2)[3], const double (*v)[3], const double (*x)[3]) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = clusters_.find(c);
    if (it == clusters_.end() || n < 0) {
        err = "resident: bad cluster or count";
        return -1;
    }
    Cluster &cl = *it->second;
    cv_idle_.wait(lk, [&] { return cl.inflight == 0; });
    if (n == 0) return 0;
    const long long cap = cl.cap;
    long long lo = cap, hi = -1;
    for (int k = 0; k < n; ++k) {
        const long long a = address ? address[k] : k;
        if (a < 0 || a >= cap) {
            err = "resident: address beyond the cluster's capacity";
            return -1;
        }
        lo = std::min(lo, a);
        hi = std::max(hi, a);
        double *r = cl.h_raw;
        r[JF_T * cap + a] = tj[k];
        r[JF_M * cap + a] = mass[k];
        for (int q = 0; q < 3; ++q) {
            r[(JF_X + q) * cap + a] = x[k][q];
            r[(JF_V + q) * cap + a] = v[k][q];
            r[(JF_A2 + q) * cap + a] = a2[k][q];
            r[(JF_J6 + q) * cap + a] = j6[k][q];
            r[(JF_K18 + q) * cap + a] = 0.0;
            cl.xmax = std::max(cl.xmax, std::fabs(x[k][q]));
        }
    }
    cudaSetDevice(device_);
    const size_t cnt = (size_t)(hi - lo + 1);
    for (int f = 0; f < JF_COUNT; ++f)
        RES_CHECK(cudaMemcpyAsync(cl.d_raw + f * cap + lo, cl.h_raw + f * cap + lo, 8 * cnt, cudaMemcpyHostToDevice,
                                  copy_), "j upload");
    RES_CHECK(cudaStreamSynchronize(copy_), "j upload");
    return 0;
}

long long Resident::submit(int c, double ti, int nj, int ni, const int *index, const double (*xi)[3],
                           const double (*vi)[3]) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = clusters_.find(c);
    if (it == clusters_.end() || ni < 0 || nj <= 0 || !started_ || (ni > 0 && (!index || !xi || !vi))) {
        err = "resident: bad cluster, sizes or arrays";
        return -1;
    }
    Cluster &cl = *it->second;
    if (nj > cl.cap || (size_t)ni > dev_.i_cap) {
        err = "resident: call larger than the cluster or the batch workspace";
        return -1;
    }
    const long long id = head_;
    const int k = (int)(id % kResSlots);
    if (__atomic_load_n(&slots_[k].state, __ATOMIC_ACQUIRE) != kFree) {
        err = "resident: request ring full (wait for earlier calls first)";
        return -1;
    }
    SlotHost &h = host_[k];
    const size_t ibytes = sizeof(IRec) * (size_t)ni;
    h.bytes = ibytes + 60 * (size_t)ni;
    h.buf = arena_.alloc(h.bytes);
    if (!h.buf) {
        err = "resident: pinned request buffers";
        return -1;
    }
    h.irec = reinterpret_cast<IRec *>(h.buf);
    h.out = h.buf + ibytes;
    unsigned char *dbuf = arena_.device_ptr(h.buf);
    ++head_;
    double xm = cl.xmax;
    for (int i = 0; i < ni; ++i) {
        IRec &r = h.irec[i];
        for (int q = 0; q < 3; ++q) {
            r.x[q] = xi[i][q];
            r.v[q] = vi[i][q];
            xm = std::max(xm, std::fabs(xi[i][q]));
        }
        r.h2 = 0.0;
        r.index = index[i];
        r.pad = 0;
    }
    cl.xmax = xm;
    // fixed-point range: the engine's rule (2^(E-1) > |x|max, factor-2 margin), only widened
    const int E = (xm > 0 && std::isfinite(xm)) ? std::max(std::ilogb(xm) + 2, -60) : 1;
    cl.E = std::max(cl.E, E);
    ResSlot &s = slots_[k];
    s.cluster = c;
    s.ni = ni;
    s.nj = nj;
    s.ti = ti;
    s.eps2 = cl.eps2;
    s.fs = scale_of(cl.E);
    s.irec = reinterpret_cast<IRec *>(dbuf);
    s.out = dbuf + ibytes;
    s.batch = -1;
    s.batch_size = 0;
    s.status = 0;
    h.t_submit = now_s();
    h.cluster = c;
    h.id = id;
    cl.inflight++;
    if (holding_) {
        h.held = true;
        held_.push_back(id);
        return id;
    }
    h.held = false;
    __atomic_store_n(&s.state, (int)kReady, __ATOMIC_RELEASE);
    launch_locked();  // when it fails, the call is marked failed and its wait reports it
    return id;
}

void Resident::hold(bool on) {
    std::lock_guard<std::mutex> lk(mu_);
    holding_ = on;
    if (on) return;
    // Release the held calls last first: when the ring position the kernel
    // looks at turns READY, all later ones already are, so they are gathered
    // into one batch.
    for (auto it = held_.rbegin(); it != held_.rend(); ++it) {
        const int k = (int)(*it % kResSlots);
        host_[k].held = false;
        __atomic_store_n(&slots_[k].state, (int)kReady, __ATOMIC_RELEASE);
    }
    held_.clear();
    launch_locked();
}

// Kernel not running (it left after its idle time, or after an error) and a
// call waiting: launch it again.  Called with mu_ held.  When that fails,
// the calls no kernel will serve -- the READY ones, and the TAKEN ones too
// when the previous kernel died with a CUDA error -- are marked failed, so
// their waiters return and free their slots.
int Resident::launch_locked() {
    bool kernel_died = false;
    const int rc = launch_try_locked(kernel_died);
    if (rc) {
        if (kernel_died) fail_slots_locked(kTaken);
        fail_slots_locked(kReady);
        cv_idle_.notify_all();
    }
    return rc;
}

void Resident::fail_slots_locked(int state) {
    for (int k = 0; k < kResSlots; ++k)
        if (__atomic_load_n(&slots_[k].state, __ATOMIC_ACQUIRE) == state) {
            slots_[k].status |= kLostWithKernel;
            __atomic_store_n(&slots_[k].state, (int)kFailed, __ATOMIC_RELEASE);
        }
}

int Resident::launch_try_locked(bool &kernel_died) {
    if (launched_) {
        const cudaError_t q = cudaEventQuery(ev_run_);
        if (q == cudaErrorNotReady) return 0;  // running
        launched_ = false;
        if (q != cudaSuccess) {
            err = std::string("resident: kernel failed: ") + cudaGetErrorString(q);
            kernel_died = true;
            return -1;
        }
        if (__atomic_load_n(&ctl_->error, __ATOMIC_ACQUIRE)) recover_locked();
    }
    bool ready = false;
    for (int k = 0; k < kResSlots && !ready; ++k)
        ready = __atomic_load_n(&slots_[k].state, __ATOMIC_ACQUIRE) == kReady;
    if (!ready) return 0;
    cudaSetDevice(device_);
    RES_CHECK(cudaMemsetAsync(dev_.bar_count, 0, 4, stream_), "launch");
    RES_CHECK(cudaMemsetAsync(dev_.leave, 0, 4, stream_), "launch");
    ResDev d = dev_;
    void *args[] = {&d};
    void (*fn)(const ResDev) = kmode_ == kKernF64 ? resident_kernel<kKernF64> : resident_kernel<kKernMixedP>;
    const cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<void *>(fn), dim3(ctas_), dim3(256), args,
                                                      smem_, stream_);
    if (e != cudaSuccess) {
        err = std::string("resident: launch failed: ") + cudaGetErrorString(e);
        return -1;
    }
    stats_.launches++;
    const cudaError_t r = cudaEventRecord(ev_run_, stream_);
    if (r != cudaSuccess) {
        // The kernel runs but cannot be watched: wait for it to leave (it
        // serves the READY calls, then exits after its idle time), so that no
        // second kernel is launched beside it.
        err = std::string("resident: launch: ") + cudaGetErrorString(r);
        cudaStreamSynchronize(stream_);
        return 0;
    }
    launched_ = true;
    return 0;
}

// After the kernel left with an error: the calls it had taken will not
// complete; mark them failed (their waiters report it), and clear the
// i-tile arrival counters a cut-short batch may have left raised.
void Resident::recover_locked() {
    __atomic_store_n(&ctl_->error, 0u, __ATOMIC_RELEASE);
    fail_slots_locked(kTaken);
    cudaMemsetAsync(dev_.tcnt, 0, 4 * dev_.i_cap, stream_);
    stats_.recoveries++;
}

int Resident::wait(long long id, double (*acc)[3], double (*jerk)[3], double *pot, int *nn, double *latency_s,
                   long long *batch, int *batch_size) {
    const int k = (int)(id % kResSlots);
    ResSlot &s = slots_[k];
    SlotHost &h = host_[k];
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (id < 0 || h.id != id) {
            err = "resident: unknown request";
            return -1;
        }
    }
    const double t0 = now_s();
    int st;
    for (long long spin = 0;; ++spin) {
        st = __atomic_load_n(&s.state, __ATOMIC_ACQUIRE);
        if (st == kDone || st == kFailed) break;
        if ((spin & 1023) == 1023) {
            std::lock_guard<std::mutex> lk(mu_);
            if (!h.held) launch_locked();  // a failed launch fails this call: the loop then ends
            if (now_s() - t0 > 600.0) {
                err = "resident: call not served within 600 s";
                return -3;
            }
        }
        // spin briefly, then yield, then nap (many client threads may wait at once)
        if (spin > 20000)
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        else if (spin > 2048)
            std::this_thread::yield();
    }
    const double t_done = now_s();
    const int ni = s.ni;
    int rc = 0;
    if (st == kFailed) {
        rc = (s.status & kLostWithKernel) ? 2 : -1;
        err = rc == 2 ? "resident: the serving kernel left with an error before the call completed"
                      : "resident: call larger than the batch workspace";
    } else if (s.status & ST_TMA_TIMEOUT) {
        rc = 3;
        err = "resident: j-tile copy wait timed out on the device";
    } else if (s.status & ST_RANGE) {
        rc = 4;
        err = "resident: positions outside the fixed-point range (widened; submit again)";
    } else {
        const double *o = reinterpret_cast<const double *>(h.out);
        if (acc) memcpy(acc, o, 24 * (size_t)ni);
        if (jerk) memcpy(jerk, o + 3 * (size_t)ni, 24 * (size_t)ni);
        if (pot) memcpy(pot, o + 6 * (size_t)ni, 8 * (size_t)ni);
        if (nn) memcpy(nn, reinterpret_cast<const int *>(o + 7 * (size_t)ni), 4 * (size_t)ni);
    }
    if (latency_s) *latency_s = t_done - h.t_submit;
    if (batch) *batch = s.batch;
    if (batch_size) *batch_size = s.batch_size;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = clusters_.find(h.cluster);
        if (it != clusters_.end()) {
            it->second->inflight--;
            if (rc == 4) it->second->E += 2;  // a wider grid for the caller's next submit
        }
        h.id = -1;
        arena_.release(h.buf, h.bytes);
        h.buf = nullptr;
        __atomic_store_n(&s.state, (int)kFree, __ATOMIC_RELEASE);
    }
    cv_idle_.notify_all();
    return rc;
}

}  // namespace g6

// ---------------------------------------------------------------------------
#pragma GCC visibility push(default)
#include "../../include/g6b200.h"
#pragma GCC visibility pop

struct g6b200_resident {
    g6::Resident *r;
};

extern "C" {

__attribute__((visibility("default"))) g6b200_resident *g6b200_res_create(int device, long long hbm_budget_bytes,
                                                                         int precision, int max_batch) {
    auto *r = new g6::Resident(device, hbm_budget_bytes, precision, max_batch);
    if (r->start()) {
        g6::record_error(r->err);
        delete r;
        return nullptr;
    }
    return new g6b200_resident{r};
}

__attribute__((visibility("default"))) int g6b200_res_open_cluster(g6b200_resident *h, long long n_cap,
                                                                   double eps2) {
    const int rc = h->r->open_cluster(n_cap, eps2);
    if (rc < 0) g6::record_error(h->r->err);
    return rc;
}

__attribute__((visibility("default"))) int g6b200_res_close_cluster(g6b200_resident *h, int cluster) {
    return h->r->close_cluster(cluster);
}

__attribute__((visibility("default"))) int g6b200_res_set_j(g6b200_resident *h, int cluster, int n,
                                                            const int *address, const double *tj,
                                                            const double *mass, const double (*j6)[3],
                                                            const double (*a2)[3], const double (*v)[3],
                                                            const double (*x)[3]) {
    const int rc = h->r->set_j(cluster, n, address, tj, mass, j6, a2, v, x);
    if (rc) g6::record_error(h->r->err);
    return rc;
}

__attribute__((visibility("default"))) long long g6b200_res_submit(g6b200_resident *h, int cluster, double ti,
                                                                   int nj, int ni, const int *index,
                                                                   const double (*xi)[3], const double (*vi)[3]) {
    const long long id = h->r->submit(cluster, ti, nj, ni, index, xi, vi);
    if (id < 0) g6::record_error(h->r->err);
    return id;
}

__attribute__((visibility("default"))) int g6b200_res_wait(g6b200_resident *h, long long request,
                                                           double (*acc)[3], double (*jerk)[3], double *pot,
                                                           int *nn, double *latency_s, long long *batch,
                                                           int *batch_size) {
    const int rc = h->r->wait(request, acc, jerk, pot, nn, latency_s, batch, batch_size);
    if (rc) g6::record_error(h->r->err);
    return rc;
}

__attribute__((visibility("default"))) void g6b200_res_hold(g6b200_resident *h, int hold) { h->r->hold(hold != 0); }

__attribute__((visibility("default"))) void g6b200_res_selftest_stall(g6b200_resident *h) { h->r->selftest_stall(); }

__attribute__((visibility("default"))) int g6b200_res_stats(g6b200_resident *h, g6b200_res_stats_t *out) {
    const g6::ResStats s = h->r->stats();
    out->batches = s.batches;
    out->calls = s.calls;
    out->launches = s.launches;
    out->recoveries = s.recoveries;
    out->max_batch = s.max_batch;
    return 0;
}

__attribute__((visibility("default"))) void g6b200_res_destroy(g6b200_resident *h) {
    if (!h) return;
    delete h->r;
    delete h;
}

}  // extern "C"
