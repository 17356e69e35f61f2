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
