// nblist.cu -- neighbour-list compaction.
//
// The force kernel appends hits {j : |x_j - x_i|^2 < h2_i} per i with an
// atomic cursor (order depends on scheduling).  These two kernels make the
// result deterministic and compact: an exclusive scan of the clamped counts,
// then one CTA per i sorting its list ascending (bitonic sort in shared
// memory) into the compacted output.  Ascending address order is what the
// CPU loop produces (daughters in order) and what kira's nn/coll recompute
// over the list relies on for first-index tie breaking
// (hdyn_grape6.C:2430-2456, update_nn_coll).
#include <climits>
#include "common.cuh"
#include "kernels.h"

namespace g6 {

// One CTA of 1024 threads; each thread scans a contiguous run of counts.
__global__ void __launch_bounds__(1024) nb_scan_kernel(int ni, const int *__restrict__ count, int cap,
                                                       long long *__restrict__ offsets) {
    __shared__ long long part[1024];
    const int t = threadIdx.x;
    const int per = (ni + 1023) / 1024;
    const int b = t * per;
    const int e = min(b + per, ni);
    long long local = 0;
    for (int i = b; i < e; ++i) local += min(count[i], cap);
    part[t] = local;
    __syncthreads();
    // Hillis-Steele inclusive scan over 1024 partial sums.
    for (int off = 1; off < 1024; off <<= 1) {
        long long v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = t > 0 ? part[t - 1] : 0;
    for (int i = b; i < e; ++i) {
        offsets[i] = run;
        run += min(count[i], cap);
    }
    if (t == 1023) offsets[ni] = part[1023];
}

// One CTA per i.  Dynamic shared memory: next_pow2(cap) ints.
__global__ void nb_sort_kernel(const int *__restrict__ count, const int *__restrict__ list, int cap,
                               const long long *__restrict__ offsets, int *__restrict__ out) {
    extern __shared__ int keys[];
    const int i = blockIdx.x;
    const int n = min(count[i], cap);
    if (n <= 0) return;
    const int *src = list + (size_t)i * cap;
    int *dst = out + offsets[i];
    if (n == 1) {
        if (threadIdx.x == 0) dst[0] = src[0];
        return;
    }
    int m = 1;
    while (m < n) m <<= 1;
    for (int k = threadIdx.x; k < m; k += blockDim.x) keys[k] = k < n ? src[k] : INT_MAX;
    __syncthreads();
    for (int size = 2; size <= m; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int k = threadIdx.x; k < m; k += blockDim.x) {
                const int o = k ^ stride;
                if (o > k) {
                    const bool up = (k & size) == 0;
                    const int a = keys[k], b = keys[o];
                    if ((a > b) == up) {
                        keys[k] = b;
                        keys[o] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = keys[k];
}

// Full neighbour list of one GRAPE-4 i-particle over the predicted FP64
// j-set, for lists longer than the per-i capacity of the force kernel's
// lists (the GRAPE-4 readout h3nblist_ has no length limit).  One CTA of
// 1024 threads walks the addresses in order; each chunk's hits are placed by
// a ballot prefix, so the list comes out ascending.  The test is the force
// kernel's (g4_r2 < h2_i).  Writes at most cap entries; *count gets the
// number of hits.
__global__ void __launch_bounds__(1024) nb_full_g4_kernel(const JRecF64 *__restrict__ jrec, int nj, IRec q,
                                                          double eps2, int *__restrict__ out, int cap,
                                                          int *__restrict__ count) {
    __shared__ int warp_hits[32];
    __shared__ int base;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (int j0 = 0; j0 < nj; j0 += blockDim.x) {
        const int j = j0 + threadIdx.x;
        bool hit = false;
        if (j < nj) {
            const double4 p = jrec[j].pos;
            hit = g4_r2(p.x - q.x[0], p.y - q.x[1], p.z - q.x[2], eps2) < q.h2;
        }
        const unsigned b = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) warp_hits[w] = __popc(b);
        __syncthreads();
        int off = base;
        for (int k = 0; k < w; ++k) off += warp_hits[k];
        if (hit) {
            const int pos = off + __popc(b & ((1u << lane) - 1u));
            if (pos < cap) out[pos] = j;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int k = 0; k < nw; ++k) t += warp_hits[k];
            base += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = base;
}

cudaError_t launch_nb_full_g4(cudaStream_t s, const void *jrec, int nj, const IRec &q, double eps2, int *out,
                              int cap, int *count) {
    nb_full_g4_kernel<<<1, 1024, 0, s>>>(reinterpret_cast<const JRecF64 *>(jrec), nj, q, eps2, out, cap, count);
    return cudaGetLastError();
}

cudaError_t launch_nb_compact(cudaStream_t s, int ni, const int *count, const int *list, int cap,
                              long long *offsets, int *out) {
    if (ni <= 0) return cudaSuccess;
    nb_scan_kernel<<<1, 1024, 0, s>>>(ni, count, cap, offsets);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int m = 1;
    while (m < cap) m <<= 1;
    nb_sort_kernel<<<ni, 256, m * sizeof(int), s>>>(count, list, cap, offsets, out);
    return cudaGetLastError();
}

}  // namespace g6
