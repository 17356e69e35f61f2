// split.cu -- one cluster's j-set split across GPUs: order-independent
// combination of the per-rank partial sums on the device.
//
// The reference's distributed force (kira_ev.C:275-420, under -DUSEMPI)
// gives each rank a contiguous range of j, computes every i's partial sums
// over it and combines them with MPI_Allreduce: SUM for acc/jerk/pot
// (kira_ev.C:327-328) and MINLOC for the nearest neighbour (:409-410).  An
// FP64 SUM depends on how the j-set is cut, so results change with the rank
// count.  Here the j-set is cut into global blocks of a fixed size; each
// block's FP64 partial (one split of the force kernel, computed the same way
// on whichever rank holds the block) is converted to 64-bit fixed point on a
// per-(i, quantity) scale all ranks agree on, and the fixed-point values are
// summed exactly -- so the result is bit-identical for any number of ranks.
//
// Three steps, with a collective after each of the first two (the caller
// runs them, e.g. NCCL all_reduce on device buffers):
//   1. split_agree:  agree[8 ni] int64 = per (i, q) the exponent e with
//                    |partial| < 2^e over this rank's blocks (q = acc x/y/z,
//                    jerk x/y/z, pot), and -(bits of the smallest nn r^2);
//                    -> all_reduce MAX (largest exponent, smallest r^2).
//   2. split_fix:    sums[7 ni] int64 = sum over this rank's blocks of
//                    rint(partial * 2^(62 - g - e)), g = ceil(log2(blocks));
//                    negj[ni] = -(smallest global j of a block whose nn r^2
//                    equals the agreed minimum), or -INT64_MAX;
//                    -> all_reduce SUM (sums), MAX (negj).
//   3. split_finish: FP64 results = sums * 2^-(62 - g - e); nn = -negj.
// Each |term| < 2^(62 - g) and there are at most 2^g blocks, so the int64
// sums cannot overflow.
#include <cstdint>
#include "common.cuh"
#include "kernels.h"

namespace g6 {

namespace {

constexpr int kQ = 7;                       // acc x/y/z, jerk x/y/z, pot
constexpr long long kNoExp = -(1LL << 40);  // no nonzero partial

__device__ __forceinline__ double q_of(const Partial &p, int q) {
    return q < 3 ? p.acc[q] : (q < 6 ? p.jerk[q - 3] : p.pot);
}

__device__ __forceinline__ long long exp_of(double x) {
    if (x == 0.0) return kNoExp;
    int e;
    frexp(x, &e);  // |x| = f 2^e, f in [0.5, 1): |x| < 2^e
    return e;
}

__global__ void split_agree_kernel(int ni, int nsplit, const Partial *__restrict__ part,
                                   long long *__restrict__ agree) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ni) return;
    long long e[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) e[q] = kNoExp;
    double r2 = __longlong_as_double(0x7ff0000000000000LL);  // +inf: no candidate
    for (int s = 0; s < nsplit; ++s) {
        const Partial p = part[(size_t)s * ni + i];
#pragma unroll
        for (int q = 0; q < kQ; ++q) e[q] = max(e[q], exp_of(q_of(p, q)));
        if (p.nn_j >= 0 && p.nn_r2 < r2) r2 = p.nn_r2;
    }
#pragma unroll
    for (int q = 0; q < kQ; ++q) agree[(size_t)q * ni + i] = e[q];
    agree[(size_t)kQ * ni + i] = -__double_as_longlong(r2);  // r2 >= 0: bits order like the values
}

__global__ void split_fix_kernel(int ni, int nsplit, int g, long long j_offset, const Partial *__restrict__ part,
                                 const long long *__restrict__ agree, long long *__restrict__ sums,
                                 long long *__restrict__ negj) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ni) return;
    int sc[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
        const long long e = agree[(size_t)q * ni + i];
        sc[q] = e == kNoExp ? 0 : (int)(62 - g - e);
    }
    const double r2min = __longlong_as_double(-agree[(size_t)kQ * ni + i]);
    long long acc[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) acc[q] = 0;
    long long best = INT64_MAX;
    for (int s = 0; s < nsplit; ++s) {
        const Partial p = part[(size_t)s * ni + i];
#pragma unroll
        for (int q = 0; q < kQ; ++q) acc[q] += __double2ll_rn(ldexp(q_of(p, q), sc[q]));
        if (p.nn_j >= 0 && p.nn_r2 == r2min) best = min(best, (long long)p.nn_j + j_offset);
    }
#pragma unroll
    for (int q = 0; q < kQ; ++q) sums[(size_t)q * ni + i] = acc[q];
    negj[i] = -best;
}

__global__ void split_finish_kernel(int ni, int g, long long nj_total, const long long *__restrict__ agree,
                                    const long long *__restrict__ sums, const long long *__restrict__ negj,
                                    double *__restrict__ out_acc, double *__restrict__ out_jerk,
                                    double *__restrict__ out_pot, int *__restrict__ out_nn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ni) return;
    double v[kQ];
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
        const long long e = agree[(size_t)q * ni + i];
        v[q] = e == kNoExp ? 0.0 : ldexp(__ll2double_rn(sums[(size_t)q * ni + i]), -(int)(62 - g - e));
    }
    for (int c = 0; c < 3; ++c) {
        out_acc[3 * (size_t)i + c] = v[c];
        out_jerk[3 * (size_t)i + c] = v[3 + c];
    }
    out_pot[i] = v[6];
    const long long j = -negj[i];
    out_nn[i] = (j < 0 || j >= nj_total) ? 0 : (int)j;
}

}  // namespace

int split_log2_blocks(long long nblocks) {
    int g = 0;
    while ((1LL << g) < nblocks) ++g;
    return g;
}

void launch_split_agree(cudaStream_t s, int ni, int nsplit, const Partial *part, long long *agree) {
    if (ni > 0) split_agree_kernel<<<(ni + 255) / 256, 256, 0, s>>>(ni, nsplit, part, agree);
}

void launch_split_fix(cudaStream_t s, int ni, int nsplit, int g, long long j_offset, const Partial *part,
                      const long long *agree, long long *sums, long long *negj) {
    if (ni > 0) split_fix_kernel<<<(ni + 255) / 256, 256, 0, s>>>(ni, nsplit, g, j_offset, part, agree, sums, negj);
}

void launch_split_finish(cudaStream_t s, int ni, int g, long long nj_total, const long long *agree,
                         const long long *sums, const long long *negj, double *acc, double *jerk, double *pot,
                         int *nn) {
    if (ni > 0)
        split_finish_kernel<<<(ni + 255) / 256, 256, 0, s>>>(ni, g, nj_total, agree, sums, negj, acc, jerk, pot, nn);
}

}  // namespace g6
