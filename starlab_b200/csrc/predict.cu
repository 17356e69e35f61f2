// predict.cu -- j-memory scatter and the j-particle predictor.
//
// The GRAPE-6 board predicted every j-particle to the block time on board
// (the CPU equivalent is _dyn_::predict_loworder, include/_dyn_.h:265-299);
// here one thread per j reads the FP64 SoA j-state (coalesced) and writes
// one AoS record per j in the precision mode's layout (common.cuh).  The
// kernel is HBM-bound: 104 B read + 48 B (mixed) or 64 B (FP64) written
// per j.
#include "common.cuh"
#include "kernels.h"
#include "predict_device.cuh"

namespace g6 {

// Host staging records -> raw j-state.  One thread per (record, field):
// reads are contiguous, writes land in 17 SoA rows.
__global__ void scatter_j_kernel(int n, const int *__restrict__ addr,
                                 const int *__restrict__ index,
                                 const double *__restrict__ vals,
                                 double *__restrict__ jraw, int *__restrict__ jindex,
                                 int cap) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long total = (long long)n * JF_COUNT;
    if (t < total) {
        int r = (int)(t / JF_COUNT);
        int f = (int)(t - (long long)r * JF_COUNT);
        int a = addr[r];
        jraw[(size_t)f * cap + a] = vals[t];
        if (f == 0) jindex[a] = index[r];
    }
}

// Bulk upload: the caller's arrays, copied as they are (t[n], m[n], x, v,
// a2, j6, k18 as [n][3]), scattered into the raw j-state.  One thread per
// (field, particle), so a warp writes one SoA row contiguously when the
// addresses are.
__global__ void scatter_bulk_kernel(int n, BulkJ b, double *__restrict__ jraw, int *__restrict__ jindex, int cap) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * JF_COUNT) return;
    const int f = (int)(t / n);
    const int r = (int)(t - (long long)f * n);
    const int a = b.addr ? b.addr[r] : r;
    double val;
    if (f == JF_T) {
        val = b.t[r];
    } else if (f == JF_M) {
        val = b.m[r];
    } else {
        const int g = (f - JF_X) / 3, c = (f - JF_X) % 3;  // x, v, a2, j6, k18 rows follow each other
        const double *src = g == 0 ? b.x : g == 1 ? b.v : g == 2 ? b.a2 : g == 3 ? b.j6 : b.k18;
        val = src ? src[3 * (size_t)r + c] : 0.0;
    }
    jraw[(size_t)f * cap + a] = val;
    if (f == JF_T) jindex[a] = b.index ? b.index[r] : a;
}

__global__ void predict_mixed_kernel(const double *__restrict__ jraw, const int *__restrict__ jindex,
                                     int cap, int nj, int nj_pad, double ti, FixedScale fs,
                                     JRecMixed *__restrict__ out, unsigned *__restrict__ status) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nj_pad) return;
    JRecMixed r;
    if (j < nj) {
        double xp[3], vp[3], m;
        predict_one(jraw, cap, j, ti, xp, vp, m);
        float hi[3], lo[3];
        bool bad = false;
#pragma unroll
        for (int c = 0; c < 3; c++) bad |= !to_fixed_split(xp[c], fs, hi[c], lo[c]);
        if (bad) atomicOr(status, ST_RANGE);
        r.hi = make_float4(hi[0], hi[1], hi[2], (float)m);
        r.lo = make_float4(lo[0], lo[1], lo[2], __int_as_float(jindex[j]));
        r.vel = make_float4((float)vp[0], (float)vp[1], (float)vp[2], 0.f);
    } else {
        r.hi = make_float4(kDummyPos, kDummyPos, kDummyPos, 0.f);
        r.lo = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        r.vel = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    out[j] = r;
}

// One thread per pair of consecutive j (paired layout, JPairMixed).
__global__ void predict_pair_kernel(const double *__restrict__ jraw, const int *__restrict__ jindex,
                                    int cap, int nj, int nj_pad, double ti, FixedScale fs,
                                    JPairMixed *__restrict__ out, unsigned *__restrict__ status) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * q >= nj_pad) return;
    predict_pair_unit(jraw, jindex, cap, nj, q, ti, fs, out, status);
}

__global__ void predict_f64_kernel(const double *__restrict__ jraw, const int *__restrict__ jindex,
                                   int cap, int nj, int nj_pad, double ti,
                                   JRecF64 *__restrict__ out) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nj_pad) return;
    predict_f64_unit(jraw, jindex, cap, nj, j, ti, out);
}

// i-records for a self-gravity sweep: the i-particles are j-addresses
// [i0, i0 + ni), predicted to ti in FP64 exactly as the j-side is.
__global__ void irec_from_j_kernel(const double *__restrict__ jraw, const int *__restrict__ jindex,
                                   int cap, int i0, int ni, double ti, IRec *__restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ni) return;
    int j = i0 + k;
    double xp[3], vp[3], m;
    predict_one(jraw, cap, j, ti, xp, vp, m);
    IRec r;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        r.x[c] = xp[c];
        r.v[c] = vp[c];
    }
    r.h2 = 0.0;
    r.index = jindex[j];
    r.pad = 0;
    out[k] = r;
}

// ---- small calls: updates + prediction + i-records in one launch

__device__ __forceinline__ void predict_vals(const double *v17, double ti, double xp[3], double vp[3], double &m) {
    const double dt = ti - v17[JF_T];
    m = v17[JF_M];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const double x = v17[JF_X + c], v = v17[JF_V + c], a2 = v17[JF_A2 + c], j6 = v17[JF_J6 + c];
        xp[c] = x + dt * (v + dt * (a2 + dt * j6));
        vp[c] = v + dt * (2.0 * a2 + dt * (3.0 * j6));
    }
}

// Position of address j in the ascending update list, or -1.
__device__ __forceinline__ int find_update(const int *addr, int n, int j) {
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int a = addr[mid];
        if (a == j) return mid;
        if (a < j) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

// Predicted j (or a dummy beyond nj): the update's values when j is being
// updated (its raw state is rewritten by another thread of this launch),
// the raw j-state otherwise.
__device__ __forceinline__ bool small_pred(const SmallCall &sc, const int *s_addr, const double *jraw,
                                           const int *jindex, int j, double xp[3], double vp[3], double &m,
                                           int &id) {
    if (j >= sc.nj) return false;
    const int s = find_update(s_addr, sc.n_upd, j);
    if (s >= 0) {
        predict_vals(sc.vals[s], sc.ti, xp, vp, m);
        id = sc.index[s];
    } else {
        predict_one(jraw, sc.cap, j, sc.ti, xp, vp, m);
        id = jindex[j];
    }
    return true;
}

template <int KM>
__global__ void __launch_bounds__(256) small_call_kernel(const __grid_constant__ SmallCall sc,
                                                         double *__restrict__ jraw, int *__restrict__ jindex,
                                                         void *__restrict__ jrec, IRec *__restrict__ irec,
                                                         double *__restrict__ ieps2, unsigned *__restrict__ status2) {
    __shared__ int s_addr[kSmallMax];
    const int tid = threadIdx.x;
    if (tid < sc.n_upd) s_addr[tid] = sc.addr[tid];
    if (blockIdx.x == 0) {
        if (tid < sc.ni) {
            irec[tid] = sc.irec[tid];
            if (sc.g4) ieps2[tid] = sc.ieps2[tid];
        }
        if (tid == 0) status2[sc.parity ^ 1] = 0u;
        if (tid < sc.n_upd) {  // persist the updates (no thread of this launch reads these addresses' raw state)
            const int a = sc.addr[tid];
#pragma unroll
            for (int f = 0; f < JF_COUNT; ++f) jraw[(size_t)f * sc.cap + a] = sc.vals[tid][f];
            jindex[a] = sc.index[tid];
        }
    }
    __syncthreads();
    if (!sc.predict) return;
    const int q = blockIdx.x * blockDim.x + tid;
    if constexpr (KM == kKernF64) {
        const int j = q;
        if (j >= sc.nj_pad) return;
        JRecF64 r;
        double xp[3], vp[3], m;
        int id;
        if (small_pred(sc, s_addr, jraw, jindex, j, xp, vp, m, id)) {
            r.pos = make_double4(xp[0], xp[1], xp[2], m);
            r.vel = make_double4(vp[0], vp[1], vp[2], (double)id);
        } else {
            r.pos = make_double4(kDummyPos, kDummyPos, kDummyPos, 0.0);
            r.vel = make_double4(0.0, 0.0, 0.0, -1.0);
        }
        reinterpret_cast<JRecF64 *>(jrec)[j] = r;
    } else if constexpr (KM == kKernMixedDS) {
        const int j = q;
        if (j >= sc.nj_pad) return;
        JRecMixed r;
        double xp[3], vp[3], m;
        int id;
        if (small_pred(sc, s_addr, jraw, jindex, j, xp, vp, m, id)) {
            float hi[3], lo[3];
            bool bad = false;
#pragma unroll
            for (int c = 0; c < 3; c++) bad |= !to_fixed_split(xp[c], sc.fs, hi[c], lo[c]);
            if (bad) atomicOr(&status2[sc.parity], ST_RANGE);
            r.hi = make_float4(hi[0], hi[1], hi[2], (float)m);
            r.lo = make_float4(lo[0], lo[1], lo[2], __int_as_float(id));
            r.vel = make_float4((float)vp[0], (float)vp[1], (float)vp[2], 0.f);
        } else {
            r.hi = make_float4(kDummyPos, kDummyPos, kDummyPos, 0.f);
            r.lo = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
            r.vel = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        reinterpret_cast<JRecMixed *>(jrec)[j] = r;
    } else {
        if (2 * q >= sc.nj_pad) return;
        float hi[2][3], lo[2][3], v[2][3], m[2];
        int id[2];
        bool bad = false;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            double xp[3], vp[3], mm;
            if (small_pred(sc, s_addr, jraw, jindex, 2 * q + u, xp, vp, mm, id[u])) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    bad |= !to_fixed_split(xp[c], sc.fs, hi[u][c], lo[u][c]);
                    v[u][c] = (float)vp[c];
                }
                m[u] = (float)mm;
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
        if (bad) atomicOr(&status2[sc.parity], ST_RANGE);
        JPairMixed r;
        r.hxy = make_float4(hi[0][0], hi[1][0], hi[0][1], hi[1][1]);
        r.hzm = make_float4(hi[0][2], hi[1][2], -0.125f * m[0], -0.125f * m[1]);  // -m/8: see JPairMixed
        r.lxy = make_float4(lo[0][0], lo[1][0], lo[0][1], lo[1][1]);
        r.lzi = make_float4(lo[0][2], lo[1][2], __int_as_float(id[0]), __int_as_float(id[1]));
        r.vxy = make_float4(v[0][0], v[1][0], v[0][1], v[1][1]);
        r.vz = make_float4(v[0][2], v[1][2], 0.f, 0.f);
        reinterpret_cast<JPairMixed *>(jrec)[q] = r;
    }
}

void launch_small_call(cudaStream_t s, int kmode, const SmallCall &sc, double *jraw, int *jindex, void *jrec,
                       IRec *irec, double *ieps2, unsigned *status2) {
    const int per = kmode == kKernMixedP ? 2 : 1;
    const int units = sc.predict ? (sc.nj_pad + per - 1) / per : 1;
    const int blocks = (units + 255) / 256 > 0 ? (units + 255) / 256 : 1;
    if (kmode == kKernF64)
        small_call_kernel<kKernF64><<<blocks, 256, 0, s>>>(sc, jraw, jindex, jrec, irec, ieps2, status2);
    else if (kmode == kKernMixedDS)
        small_call_kernel<kKernMixedDS><<<blocks, 256, 0, s>>>(sc, jraw, jindex, jrec, irec, ieps2, status2);
    else
        small_call_kernel<kKernMixedP><<<blocks, 256, 0, s>>>(sc, jraw, jindex, jrec, irec, ieps2, status2);
}

void launch_irec_from_j(cudaStream_t s, const double *jraw, const int *jindex, int cap, int i0, int ni,
                        double ti, IRec *out) {
    if (ni <= 0) return;
    irec_from_j_kernel<<<(ni + 255) / 256, 256, 0, s>>>(jraw, jindex, cap, i0, ni, ti, out);
}

void launch_scatter(cudaStream_t s, int n, const int *addr, const int *index, const double *vals,
                    double *jraw, int *jindex, int cap) {
    if (n <= 0) return;
    long long total = (long long)n * JF_COUNT;
    int threads = 256;
    unsigned blocks = (unsigned)((total + threads - 1) / threads);
    scatter_j_kernel<<<blocks, threads, 0, s>>>(n, addr, index, vals, jraw, jindex, cap);
}

void launch_scatter_bulk(cudaStream_t s, int n, const BulkJ &b, double *jraw, int *jindex, int cap) {
    if (n <= 0) return;
    const long long total = (long long)n * JF_COUNT;
    const int threads = 256;
    scatter_bulk_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, s>>>(n, b, jraw, jindex, cap);
}

void launch_predict(cudaStream_t s, int kmode, const double *jraw, const int *jindex, int cap,
                    int nj, int nj_pad, double ti, const FixedScale &fs, void *jrec,
                    unsigned *status) {
    if (nj_pad <= 0) return;
    int threads = 256;
    int blocks = (nj_pad + threads - 1) / threads;
    if (kmode == kKernMixedDS)
        predict_mixed_kernel<<<blocks, threads, 0, s>>>(jraw, jindex, cap, nj, nj_pad, ti, fs,
                                                         (JRecMixed *)jrec, status);
    else if (kmode == kKernMixedP)
        predict_pair_kernel<<<(nj_pad / 2 + threads - 1) / threads, threads, 0, s>>>(
            jraw, jindex, cap, nj, nj_pad, ti, fs, (JPairMixed *)jrec, status);
    else
        predict_f64_kernel<<<blocks, threads, 0, s>>>(jraw, jindex, cap, nj, nj_pad, ti,
                                                       (JRecF64 *)jrec);
}

}  // namespace g6
