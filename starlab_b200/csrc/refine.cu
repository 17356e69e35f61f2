// refine.cu -- the mixed mode's FP64 refinement of ill-conditioned particles.
//
// Mixed-mode pair terms carry FP32 rounding (a few 1e-7 of each term).  A
// particle whose acceleration is the small remainder of large, nearly
// cancelling terms -- one dominant neighbour or massive star against the
// rest of the cluster -- then has a relative error of that size times the
// ratio of the dominant terms to the total.  The paired kernel tracks two
// indicators per i, the largest single terms qa = max m/r^2 and qj = max
// m/r^3; measured on the N = 262144 Plummer/Salpeter sweep against the FP64
// engine, every particle whose acc error exceeds 0.4e-6 has qa/|a| >= 1.2
// and every one whose jerk error exceeds 4e-6 has qj v_rms/|jerk| >= 2.0
// (v_rms: rms speed of the j-set).  A particle is flagged when qa/|a| >
// kRefineA or qj v_rms/|jerk| > kRefineJ (about 2% of a Plummer sphere) and
// recomputed with the FP64 kernel against FP64 j-records of the same block
// time; its results replace the mixed ones.
// Everything stays on the device, in two launches: flagging and compaction
// (the flag kernel's last block builds the FP64 pass's work item, its size
// read on the device by the batched kernel), and the FP64 pass, which
// writes the flagged particles' rows of the call's outputs (out_map).
#include <cmath>
#include "common.cuh"
#include "kernels.h"

namespace g6 {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double block_sum(double a) {
    __shared__ double sa[kThreads];
    sa[threadIdx.x] = a;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sa[threadIdx.x] += sa[threadIdx.x + w];
        __syncthreads();
    }
    return sa[0];
}

// sum of |v|^2 over the raw j-state, fixed order: kRefineBlocks partials,
// then one block.
__global__ void __launch_bounds__(kThreads) v2_blocks_kernel(const double *__restrict__ jraw, int cap, int nj,
                                                             double *__restrict__ work) {
    double s = 0;
    for (int j = blockIdx.x * kThreads + threadIdx.x; j < nj; j += kRefineBlocks * kThreads) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = jraw[(size_t)(JF_V + c) * cap + j];
            s += v * v;
        }
    }
    s = block_sum(s);
    if (threadIdx.x == 0) work[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) v2_total_kernel(double *work, int nj) {
    double s = 0;
    for (int b = threadIdx.x; b < kRefineBlocks; b += kThreads) s += work[b];
    s = block_sum(s);
    if (threadIdx.x == 0) work[kRefineBlocks] = nj > 0 ? s / nj : 0.0;  // mean |v|^2
}

// One FP64 work item for the flagged particles, sized by their count
// (tasks wanted: refine_tasks_wanted).  The item writes its results straight
// into the flagged particles' rows of the call's outputs (out_map = the
// flag list).
__device__ void make_refine_item(ForceParams p, ForceConfig cfg, int count, ForceParams *items, int *pre,
                                 int *counter) {
    p.ni = count;
    cfg.nsplit = refine_tasks_wanted(p.ni, p.nj_pad);
    int nt = 0;
    batch_plan(kKernF64, cfg, p, nt);
    items[0] = p;
    pre[0] = 0;  // task0
    pre[1] = nt;
    pre[2] = 0;  // ipre
    pre[3] = p.ni;
    *counter = 0;
}

// Flag and compact the ill-conditioned particles; the last block to finish
// builds the FP64 pass's work item, then zeroes the flag count and its own
// arrival counter for the next call (the count stays readable in pre[3]).
__global__ void flag_kernel(int ni, const double *__restrict__ acc, const double *__restrict__ jerk,
                            const float *__restrict__ q, const double *__restrict__ v2, int *__restrict__ count,
                            int *__restrict__ list, const IRec *__restrict__ irec, IRec *__restrict__ irec_ref,
                            ForceParams base, ForceConfig cfg, ForceParams *__restrict__ items, int *__restrict__ pre,
                            int *__restrict__ counter, unsigned *__restrict__ done) {
    __shared__ bool s_last;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ni) {
        const double vrms = sqrt(v2[kRefineBlocks]);
        const double a2 = acc[3 * (size_t)i] * acc[3 * (size_t)i] + acc[3 * (size_t)i + 1] * acc[3 * (size_t)i + 1] +
                          acc[3 * (size_t)i + 2] * acc[3 * (size_t)i + 2];
        const double j2 = jerk[3 * (size_t)i] * jerk[3 * (size_t)i] +
                          jerk[3 * (size_t)i + 1] * jerk[3 * (size_t)i + 1] +
                          jerk[3 * (size_t)i + 2] * jerk[3 * (size_t)i + 2];
        const double qa = q[2 * (size_t)i], qj = q[2 * (size_t)i + 1];
        // flagged unless both ratios are finite and within their bounds
        const bool good = qa * qa <= kRefineA * kRefineA * a2 && qj * qj * vrms * vrms <= kRefineJ * kRefineJ * j2;
        if (!good) {
            const int k = atomicAdd(count, 1);
            list[k] = i;
            irec_ref[k] = irec[i];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    make_refine_item(base, cfg, atomicAdd(count, 0), items, pre, counter);
    *count = 0;
    *done = 0;
}

}  // namespace

void launch_refine_v2(cudaStream_t s, const double *jraw, int cap, int nj, double *work) {
    v2_blocks_kernel<<<kRefineBlocks, kThreads, 0, s>>>(jraw, cap, nj, work);
    v2_total_kernel<<<1, kThreads, 0, s>>>(work, nj);
}

cudaError_t launch_refine(cudaStream_t s, const RefineArgs &r, int num_sms) {
    const int ni = r.ni;
    if (ni <= 0) return cudaSuccess;
    ForceConfig cfg = batch_config(kKernF64);
    ForceParams base{};
    base.jrec = r.jrec64;
    base.nj = r.nj;
    base.nj_pad = r.nj_pad;
    base.irec = r.irec_ref;
    base.eps2 = r.eps2;
    base.part = r.part;
    base.out_acc = r.acc;  // rows list[k] of the call's outputs
    base.out_jerk = r.jerk;
    base.out_pot = r.pot;
    base.out_nn = r.nn;
    base.out_map = r.list;
    base.status = r.status;
    base.tile_counter = r.tcnt;  // the last CTA of an i-tile adds its splits
    flag_kernel<<<(ni + 255) / 256, 256, 0, s>>>(ni, r.acc, r.jerk, r.q, r.v2, r.count, r.list, r.irec, r.irec_ref,
                                                 base, cfg, r.items, r.pre, r.counter, r.done);
    BatchArgs a;
    a.items = r.items;
    a.task0 = r.pre;
    a.ipre = r.pre + 2;
    a.n_items = 1;
    a.H = cfg.H;
    a.counter = r.counter;
    a.one_task_per_cta = 0;
    cudaError_t e = launch_force_batch(s, kKernF64, cfg, a, batch_ctas(kKernF64, cfg, num_sms), 0, false, r.ident);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace g6
