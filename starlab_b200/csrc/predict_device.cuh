// predict_device.cuh -- the j-particle predictor per record, shared by the
// predictor kernels (predict.cu) and the resident serving kernel
// (resident.cu): 3rd-order Taylor polynomial to the block time in FP64
// (_dyn_::predict_loworder, include/_dyn_.h:265-299, in the a/2, j/6 terms
// the adaptor sends), written in the precision mode's record layout.
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace g6 {

__device__ __forceinline__ void predict_one(const double *__restrict__ jraw, int cap, int j,
                                            double ti, double xp[3], double vp[3], double &m) {
    double dt = ti - jraw[(size_t)JF_T * cap + j];
    m = jraw[(size_t)JF_M * cap + j];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double x = jraw[(size_t)(JF_X + c) * cap + j];
        double v = jraw[(size_t)(JF_V + c) * cap + j];
        double a2 = jraw[(size_t)(JF_A2 + c) * cap + j];
        double j6 = jraw[(size_t)(JF_J6 + c) * cap + j];
        xp[c] = x + dt * (v + dt * (a2 + dt * j6));
        vp[c] = v + dt * (2.0 * a2 + dt * (3.0 * j6));
    }
}

// Pair q of the paired mixed layout (j = 2q, 2q + 1); records past nj are
// far-away massless dummies.
__device__ __forceinline__ void predict_pair_unit(const double *__restrict__ jraw, const int *__restrict__ jindex,
                                                  int cap, int nj, int q, double ti, const FixedScale &fs,
                                                  JPairMixed *__restrict__ out, unsigned *__restrict__ status) {
    float hi[2][3], lo[2][3], v[2][3], m[2];
    int id[2];
    bool bad = false;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int j = 2 * q + u;
        if (j < nj) {
            double xp[3], vp[3], mm;
            predict_one(jraw, cap, j, ti, xp, vp, mm);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                bad |= !to_fixed_split(xp[c], fs, hi[u][c], lo[u][c]);
                v[u][c] = (float)vp[c];
            }
            m[u] = (float)mm;
            id[u] = jindex[j];
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                hi[u][c] = kDummyPos;
                lo[u][c] = 0.f;
                v[u][c] = 0.f;
            }
            m[u] = 0.f;
            id[u] = -1;
        }
    }
    if (bad) atomicOr(status, ST_RANGE);
    JPairMixed r;
    r.hxy = make_float4(hi[0][0], hi[1][0], hi[0][1], hi[1][1]);
    r.hzm = make_float4(hi[0][2], hi[1][2], -0.125f * m[0], -0.125f * m[1]);  // -m/8: see JPairMixed
    r.lxy = make_float4(lo[0][0], lo[1][0], lo[0][1], lo[1][1]);
    r.lzi = make_float4(lo[0][2], lo[1][2], __int_as_float(id[0]), __int_as_float(id[1]));
    r.vxy = make_float4(v[0][0], v[1][0], v[0][1], v[1][1]);
    r.vz = make_float4(v[0][2], v[1][2], 0.f, 0.f);
    out[q] = r;
}

// Record j of the FP64 layout (dummies past nj).
__device__ __forceinline__ void predict_f64_unit(const double *__restrict__ jraw, const int *__restrict__ jindex,
                                                 int cap, int nj, int j, double ti, JRecF64 *__restrict__ out) {
    JRecF64 r;
    if (j < nj) {
        double xp[3], vp[3], m;
        predict_one(jraw, cap, j, ti, xp, vp, m);
        r.pos = make_double4(xp[0], xp[1], xp[2], m);
        r.vel = make_double4(vp[0], vp[1], vp[2], (double)jindex[j]);
    } else {
        r.pos = make_double4(kDummyPos, kDummyPos, kDummyPos, 0.0);
        r.vel = make_double4(0.0, 0.0, 0.0, -1.0);
    }
    out[j] = r;
}

}  // namespace g6
