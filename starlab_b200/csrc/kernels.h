// kernels.h -- launch interfaces between the engine (host) and the kernels.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace g6 {

// Precision modes (public, g6b200_set_precision).
constexpr int kModeF64 = 0;
constexpr int kModeMixed = 1;
// Kernel layouts: the mixed mode has two record layouts with bit-identical
// pair arithmetic: one j per record (scalar FP32), or pairs of j side by
// side evaluated with FP32x2 instructions (the default).
constexpr int kKernF64 = 0;
constexpr int kKernMixedDS = 1;
constexpr int kKernMixedP = 3;

// Fixed-point scaling of the mixed mode for position exponent E
// (all |x| < 2^E): units of the coarse grid and of the fine grid.
struct FixedScale {
    double to_units;  // 2^(23-E): x * to_units = position in coarse units
    double hi_unit;   // 2^(E-23)
    double lo_unit;   // 2^(E-46)
};

// Split an FP64 position into the coarse/fine FP32 pair (see JRecMixed).
// Returns false when |x| >= 2^E (the pair is then still close to x but the
// difference of two pairs is no longer exact).
__device__ __forceinline__ bool to_fixed_split(double x, const FixedScale &fs, float &hi, float &lo) {
    double xq = x * fs.to_units;
    double fh = floor(xq);
    double rem = xq - fh;  // exact, in [0, 1)
    hi = (float)(fh * fs.hi_unit);
    lo = (float)(floor(rem * 8388608.0) * fs.lo_unit);
    return fabs(fh) <= 8388608.0;
}

struct ForceParams {
    const void *jrec;     // JRecMixed[nj_pad] or JRecF64[nj_pad]
    int nj;               // real j count (addresses [0, nj))
    int nj_pad;           // multiple of the tile size
    int jper;             // j per split (multiple of the tile size)
    int nsplit;           // gridDim.y
    const IRec *irec;     // [ni]
    int ni;
    int H;                // j-subranges per CTA (warps sharing the same i)
    double eps2;
    FixedScale fs;
    Partial *part;        // [nsplit][ni] when nsplit > 1
    double *out_acc;      // [ni][3]   (written directly when nsplit == 1)
    double *out_jerk;     // [ni][3]
    double *out_pot;      // [ni]
    int *out_nn;          // [ni]
    int *nb_count;        // [ni]       (neighbour-list variant)
    int *nb_list;         // [ni][nb_cap]
    int nb_cap;
    int include_self;
    unsigned *status;
};

struct ForceConfig {
    int il;       // i-lanes per warp (1, 8, 32)
    int r;        // i per thread (1, 2, 4; 2 and 4 only with il = 32)
    int warps;    // warps per CTA
    int H;        // j-subranges per CTA
    int nsplit;   // CTAs along j
};

void launch_scatter(cudaStream_t s, int n, const int *addr, const int *index, const double *vals,
                    double *jraw, int *jindex, int cap);
void launch_predict(cudaStream_t s, int kmode, const double *jraw, const int *jindex, int cap,
                    int nj, int nj_pad, double ti, const FixedScale &fs, void *jrec,
                    unsigned *status);

void launch_irec_from_j(cudaStream_t s, const double *jraw, const int *jindex, int cap, int i0, int ni,
                        double ti, IRec *out);

// kmode: kKernF64 / kKernMixedDS / kKernMixedP.
int tile_size(int kmode);
size_t jrec_bytes(int kmode);
// Choose a launch configuration for ni x nj (heuristic; autotuner overrides).
ForceConfig choose_config(int kmode, int ni, int nj_pad, int num_sms, bool nb);
// Launch force (+ split reduction).  Returns a cudaError_t.
cudaError_t launch_force(cudaStream_t s, int kmode, const ForceConfig &cfg, ForceParams p,
                         bool ident, bool nb);
size_t partial_bytes(const ForceConfig &cfg, int ni);

// Neighbour lists: per-i sort + compaction into ascending address order.
// offsets[ni+1] (exclusive scan of min(count, cap)), out[total].
cudaError_t launch_nb_compact(cudaStream_t s, int ni, const int *count, const int *list, int cap,
                              long long *offsets, int *out);

}  // namespace g6
