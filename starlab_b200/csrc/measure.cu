// measure.cu -- the FP32 issue rate this GPU actually sustains, measured.
//
// The force kernel's roofline is the FP32 FMA pipe.  Instead of deriving
// its peak from the SM count and the nominal clock, this kernel measures
// it: every thread runs eight independent chains of packed FP32x2 FMAs
// (fma.rn.f32x2, the instruction the paired force kernel issues), so the
// pipe, not latency, bounds it; the FLOP rate is 2 x 2 flops per lane per
// instruction, timed with CUDA events at the clock the GPU runs at.
#include <cuda_runtime.h>
#include "../../include/g6b200.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) fp32x2_peak_kernel(float *out, float seed) {
    float2 acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = make_float2(seed + c, seed - c);
    const float2 a = make_float2(0.999999f, 0.999998f), b = make_float2(1e-7f, 2e-7f);
    for (int it = 0; it < kIters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) acc[c] = __ffma2_rn(acc[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += acc[c].x + acc[c].y;
    if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the work; never true for these inputs
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int g6b200_measure_fp32_peak(int device, double *tflops) {
    if (!tflops) return -1;
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return -1;
    float *out = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMalloc(&out, 256 * sizeof(float)) != cudaSuccess) return -1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8;  // 8 x 256 threads per SM
    fp32x2_peak_kernel<<<blocks, 256>>>(out, 1.0f);  // warm-up
    cudaEventRecord(e0);
    const int reps = 20;
    for (int r = 0; r < reps; ++r) fp32x2_peak_kernel<<<blocks, 256>>>(out, 1.0f + r);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess || ms <= 0) return -1;
    const double flops = (double)reps * blocks * 256.0 * kIters * kChains * 4.0;  // 2 lanes x FMA
    *tflops = flops / (ms * 1e-3) / 1e12;
    return 0;
}
