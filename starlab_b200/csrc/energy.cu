// energy.cu -- total energies of a potential-only sweep.
//
// The reference's energy call (grape6_calculate_energies,
// src/node/dyn/hdyn/evolve/hdyn_grape6.C:1403-1546) takes the potential of
// every particle from the engine and forms epot = sum 1/2 m_i pot_i and
// ekin = sum 1/2 m_i v_i^2 on the host.  Here both sums are formed on the
// device next to the potentials, in FP64 and in a fixed order (each block
// sums a fixed strided subset, one block adds the block sums in a fixed
// tree), so the totals are reproducible run to run.
#include "common.cuh"
#include "kernels.h"

namespace g6 {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void block_sum2(double &a, double &b) {
    __shared__ double sa[kThreads], sb[kThreads];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sa[threadIdx.x] += sa[threadIdx.x + w];
            sb[threadIdx.x] += sb[threadIdx.x + w];
        }
        __syncthreads();
    }
    a = sa[0];
    b = sb[0];
}

__global__ void __launch_bounds__(kThreads) energy_blocks_kernel(int ni, int i0, const IRec *__restrict__ irec,
                                                                 const double *__restrict__ jraw, int cap,
                                                                 const double *__restrict__ pot,
                                                                 double *__restrict__ work) {
    double ep = 0, ek = 0;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < ni; i += kEnergyBlocks * kThreads) {
        const double m = jraw[(size_t)JF_M * cap + i0 + i];
        const double vx = irec[i].v[0], vy = irec[i].v[1], vz = irec[i].v[2];
        ep += 0.5 * m * pot[i];
        ek += 0.5 * m * (vx * vx + vy * vy + vz * vz);
    }
    block_sum2(ep, ek);
    if (threadIdx.x == 0) {
        work[2 * blockIdx.x] = ep;
        work[2 * blockIdx.x + 1] = ek;
    }
}

__global__ void __launch_bounds__(kThreads) energy_total_kernel(double *work) {
    double ep = 0, ek = 0;
    for (int b = threadIdx.x; b < kEnergyBlocks; b += kThreads) {
        ep += work[2 * b];
        ek += work[2 * b + 1];
    }
    block_sum2(ep, ek);
    if (threadIdx.x == 0) {
        work[2 * kEnergyBlocks] = ep;
        work[2 * kEnergyBlocks + 1] = ek;
    }
}

}  // namespace

void launch_energy(cudaStream_t s, int ni, int i0, const IRec *irec, const double *jraw, int cap,
                   const double *pot, double *work) {
    energy_blocks_kernel<<<kEnergyBlocks, kThreads, 0, s>>>(ni, i0, irec, jraw, cap, pot, work);
    energy_total_kernel<<<1, kThreads, 0, s>>>(work);
}

}  // namespace g6
