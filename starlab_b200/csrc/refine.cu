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
// kRefineA or qj v_rms/|jerk| > kRefineJ (1-2% of a Plummer sphere) and
// recomputed with the FP64 kernel against FP64 j-records of the same block
// time; its results replace the mixed ones.
// Everything stays on the device: flagging and compaction, the item of the
// FP64 pass (its size read on the device by the batched kernel), the
// scatter of the results.
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

__global__ void flag_kernel(int ni, const double *__restrict__ acc, const double *__restrict__ jerk,
                            const float *__restrict__ q, const double *__restrict__ v2, int *__restrict__ count,
                            int *__restrict__ list, const IRec *__restrict__ irec, IRec *__restrict__ irec_ref) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ni) return;
    const double vrms = sqrt(v2[kRefineBlocks]);
    const double a2 = acc[3 * (size_t)i] * acc[3 * (size_t)i] + acc[3 * (size_t)i + 1] * acc[3 * (size_t)i + 1] +
                      acc[3 * (size_t)i + 2] * acc[3 * (size_t)i + 2];
    const double j2 = jerk[3 * (size_t)i] * jerk[3 * (size_t)i] + jerk[3 * (size_t)i + 1] * jerk[3 * (size_t)i + 1] +
                      jerk[3 * (size_t)i + 2] * jerk[3 * (size_t)i + 2];
    const double qa = q[2 * (size_t)i], qj = q[2 * (size_t)i + 1];
    // flagged unless both ratios are finite and within their bounds
    const bool good = qa * qa <= kRefineA * kRefineA * a2 && qj * qj * vrms * vrms <= kRefineJ * kRefineJ * j2;
    if (good) return;
    const int k = atomicAdd(count, 1);
    list[k] = i;
    irec_ref[k] = irec[i];
}

// One thread: the FP64 pass's single work item, sized by the flag count.
__global__ void setup_kernel(ForceParams base, ForceConfig cfg, const int *__restrict__ count,
                             ForceParams *__restrict__ items, int *__restrict__ pre, int *__restrict__ counter) {
    ForceParams p = base;
    p.ni = *count;
    int nt = 0;
    batch_plan(kKernF64, cfg, p, nt);
    items[0] = p;
    pre[0] = 0;       // task0
    pre[1] = nt;
    pre[2] = 0;       // ipre
    pre[3] = p.ni;
    *counter = 0;
}

__global__ void scatter_kernel(int ni_max, const int *__restrict__ count, const int *__restrict__ list,
                               const double *__restrict__ racc, const double *__restrict__ rjerk,
                               const double *__restrict__ rpot, const int *__restrict__ rnn, double *__restrict__ acc,
                               double *__restrict__ jerk, double *__restrict__ pot, int *__restrict__ nn) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ni_max || k >= *count) return;
    const int i = list[k];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        acc[3 * (size_t)i + c] = racc[3 * (size_t)k + c];
        jerk[3 * (size_t)i + c] = rjerk[3 * (size_t)k + c];
    }
    pot[i] = rpot[k];
    nn[i] = rnn[k];
}

}  // namespace

void launch_refine_v2(cudaStream_t s, const double *jraw, int cap, int nj, double *work) {
    v2_blocks_kernel<<<kRefineBlocks, kThreads, 0, s>>>(jraw, cap, nj, work);
    v2_total_kernel<<<1, kThreads, 0, s>>>(work, nj);
}

cudaError_t launch_refine(cudaStream_t s, const RefineArgs &r, int num_sms) {
    const int ni = r.ni;
    if (ni <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(r.count, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    flag_kernel<<<(ni + 255) / 256, 256, 0, s>>>(ni, r.acc, r.jerk, r.q, r.v2, r.count, r.list, r.irec, r.irec_ref);
    ForceConfig cfg = batch_config(kKernF64);
    ForceParams base{};
    base.jrec = r.jrec64;
    base.nj = r.nj;
    base.nj_pad = r.nj_pad;
    base.irec = r.irec_ref;
    base.eps2 = r.eps2;
    base.part = r.part;
    base.out_acc = r.racc;
    base.out_jerk = r.rjerk;
    base.out_pot = r.rpot;
    base.out_nn = r.rnn;
    base.status = r.status;
    base.tile_counter = r.tcnt;  // the last CTA of an i-tile adds its splits
    setup_kernel<<<1, 1, 0, s>>>(base, cfg, r.count, r.items, r.pre, r.counter);
    BatchArgs a;
    a.items = r.items;
    a.task0 = r.pre;
    a.ipre = r.pre + 2;
    a.n_items = 1;
    a.H = cfg.H;
    a.counter = r.counter;
    a.one_task_per_cta = 0;
    e = launch_force_batch(s, kKernF64, cfg, a, batch_ctas(kKernF64, cfg, num_sms), 0, false, r.ident);
    if (e != cudaSuccess) return e;
    scatter_kernel<<<(ni + 255) / 256, 256, 0, s>>>(ni, r.count, r.list, r.racc, r.rjerk, r.rpot, r.rnn, r.acc,
                                                    r.jerk, r.pot, r.nn);
    return cudaGetLastError();
}

size_t refine_partial_records(int ni) { return 64 * 600 + (size_t)ni; }

}  // namespace g6
