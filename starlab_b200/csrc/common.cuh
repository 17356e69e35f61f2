// common.cuh -- shared layouts and device helpers of the GRAPE-6 engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace g6 {

// ---------------------------------------------------------------------------
// j-memory layout in HBM
//
// Raw j-state, written by the scatter kernel from host updates, FP64 SoA of
// capacity `cap` (one allocation, field f at base + f*cap):
enum JField {
    JF_T = 0, JF_M = 1,
    JF_X = 2, JF_V = 5, JF_A2 = 8, JF_J6 = 11, JF_K18 = 14,
    JF_COUNT = 17
};
// plus int index[cap] (the id compared with firsthalf's index[]).
//
// Predicted j-records (one array per precision mode), AoS so that a tile of
// T consecutive j is one contiguous bulk copy into shared memory:

// Mixed mode: 48 B per j.  Positions are 47-bit fixed point on the grid
// q = 2^(E-46): hi holds the coarse part (a multiple of 2^(E-23), exact in
// FP32 for |x| < 2^E) and lo the remainder in [0, 2^(E-23)) on the fine
// grid (23 bits, exact in FP32), so (hi_j - hi_i) + (lo_j - lo_i) has both
// partial differences exact and rounds once.
struct __align__(16) JRecMixed {
    float4 hi;    // x, y, z coarse; w = mass
    float4 lo;    // x, y, z fine;   w = index (int bits)
    float4 vel;   // vx, vy, vz;     w = 0
};

// Mixed mode, paired layout: 96 B per PAIR of consecutive j (48 B per j),
// the same fixed-point split as JRecMixed with each component of the two j
// side by side, so one 8-byte half of a float4 is a ready FP32x2 operand.
struct __align__(16) JPairMixed {
    float4 hxy;   // hx0 hx1 hy0 hy1
    float4 hzm;   // hz0 hz1 -m0/8 -m1/8 (the pair kernel's Newton step yields -2/r)
    float4 lxy;   // lx0 lx1 ly0 ly1
    float4 lzi;   // lz0 lz1 index0 index1 (int bits)
    float4 vxy;   // vx0 vx1 vy0 vy1
    float4 vz;    // vz0 vz1 0 0
};

// FP64 mode: 64 B per j.
struct __align__(16) JRecF64 {
    double4 pos;  // x, y, z; w = mass
    double4 vel;  // vx, vy, vz; w = index (as double)
};

// Per-(split, i) partial sums written by the force kernel when the j-range
// is split across CTAs; reduced in split order by the reduction kernel.
struct __align__(16) Partial {
    double acc[3];
    double jerk[3];
    double pot;
    double nn_r2;
    int nn_j;
    // Error indicators of the mixed mode's refinement (0 elsewhere): the
    // largest single terms, qa = max over j of m_j / r^2, qj = max of m_j / r^3.
    float qa, qj;
    int pad;
};

// i-particle input as uploaded by firsthalf (FP64 AoS, 64 B).
struct __align__(16) IRec {
    double x[3];
    double v[3];
    double h2;
    int index;
    int pad;
};

// Far-away massless records pad the j-array to a whole number of tiles.
// At this distance r^2 ~ 3e37 stays finite in FP32 and never wins nn.
constexpr float kDummyPos = 3.0e18f;

// Device status bits (OR-ed into the per-instance status word).
enum StatusBits {
    ST_RANGE = 1,        // a predicted |x| reached 2^E (fixed-point range)
    ST_TMA_TIMEOUT = 2,  // a bulk-copy wait exceeded its bound
    ST_NB_OVERFLOW = 4,  // a neighbour list exceeded its capacity
};

// ---------------------------------------------------------------------------
// mbarrier + bulk-copy (TMA, untiled) helpers, sm_90+ PTX.

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// One bulk copy global -> shared, completing `bytes` on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: returns false (and leaves the data untouched) if the phase
// did not complete within ~limit_ns.  Never spins forever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = globaltimer_ns();
    for (unsigned it = 0; it < (1u << 30); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63) == 63 && globaltimer_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// Single-instruction approximate reciprocal square root (PTX rsqrt.approx).
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// GRAPE-4 softened squared distance, eps2 + dx^2 + dy^2 + dz^2 accumulated
// in that order (src/harpsims/harp3fastsim.c:270-272), as one fixed chain of
// fused multiply-adds so that the force kernel and the full neighbour-list
// pass round it identically (their neighbour tests then agree exactly).
__device__ __forceinline__ double g4_r2(double dx, double dy, double dz, double eps2) {
    return __fma_rn(dz, dz, __fma_rn(dy, dy, __fma_rn(dx, dx, eps2)));
}

}  // namespace g6
