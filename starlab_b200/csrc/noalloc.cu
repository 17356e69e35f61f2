// noalloc.cu -- force evaluation that allocates no memory.
//
// Some callers cannot call cudaMalloc: code that runs while another part of
// the program owns all device allocation (a host framework with its own
// memory pool or a fixed memory budget), latency-critical loops where
// cudaMalloc/cudaFree would synchronise the device, and plug-in hosts that
// hand this library only the buffers they manage.  g6b200_force_noalloc
// serves them: the caller passes device inputs and outputs, and the only
// other memory the computation needs -- the per-(j-split, i) partial sums --
// lives in one file-scope device array of fixed size, g_noalloc_scratch,
// which every GPU that loads this library holds until the process exits.
//
// The computation is the FP64 pair sum of the engine's FP64 mode
// (accumulate_acc_and_jerk, hdyn_ev.C:2019-2036; nearest neighbour without
// softening, first address on ties): the j-range is split across CTAs, each
// CTA writes its partial sums to the scratch array, and a second kernel adds
// the splits in order.  No prediction: xj/vj are taken as given.
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <mutex>
#include <string>
#include "../../include/g6b200.h"

namespace g6 {
void record_error(const std::string &msg);  // abi.cu: sets g6b200_last_error()
}

namespace {

// Scratch capacity in partial-sum records: ni * nsplit must not exceed it.
constexpr int kScratchRecords = G6B200_NOALLOC_MAX_NI;
constexpr int kTile = 128;
constexpr int kMaxDevices = 64;

struct __align__(16) NAPartial {
    double acc[3];
    double jerk[3];
    double pot;
    double nn_r2;
    int nn_j;
    int pad[3];
};

// 32768 records x 80 B = 2.5 MiB per device.
static __device__ __align__(256) NAPartial g_noalloc_scratch[kScratchRecords];

struct DeviceSetup {
    bool ready = false;
    NAPartial *scratch = nullptr;  // device address of g_noalloc_scratch
    int num_sms = 0;
};
std::mutex g_mu;
DeviceSetup g_setup[kMaxDevices];

__device__ __forceinline__ void na_take_min(double &r2, int &j, double o_r2, int o_j) {
    if (o_r2 < r2 || (o_r2 == r2 && (unsigned)o_j < (unsigned)j)) {
        r2 = o_r2;
        j = o_j;
    }
}

__global__ void __launch_bounds__(kTile) noalloc_force_kernel(
    int nj, const double *__restrict__ xj, const double *__restrict__ vj, const double *__restrict__ mj,
    int ni, const int *__restrict__ index_i, const double *__restrict__ xi, const double *__restrict__ vi,
    double eps2, int jper, int nsplit, NAPartial *__restrict__ scratch, double *__restrict__ acc,
    double *__restrict__ jerk, double *__restrict__ pot, int *__restrict__ nn) {
    __shared__ double sx[kTile], sy[kTile], sz[kTile], sm[kTile], svx[kTile], svy[kTile], svz[kTile];
    const int i = blockIdx.x * kTile + threadIdx.x;
    const bool valid = i < ni;
    double x0 = 0, y0 = 0, z0 = 0, u0 = 0, v0 = 0, w0 = 0;
    int self = -1;
    if (valid) {
        const size_t b = 3 * (size_t)i;
        x0 = xi[b]; y0 = xi[b + 1]; z0 = xi[b + 2];
        u0 = vi[b]; v0 = vi[b + 1]; w0 = vi[b + 2];
        self = index_i ? index_i[i] : -1;
    }
    double ax = 0, ay = 0, az = 0, jx = 0, jy = 0, jz = 0, p = 0;
    double best = DBL_MAX;
    int bj = -1;
    const int s = blockIdx.y;
    const int jb = s * jper;
    const int je = min(jb + jper, nj);
    for (int tb = jb; tb < je; tb += kTile) {
        const int cnt = min(kTile, je - tb);
        __syncthreads();
        if (threadIdx.x < cnt) {
            const int j = tb + threadIdx.x;
            const size_t b = 3 * (size_t)j;  // 3 j overflows int beyond 7e8 j
            sx[threadIdx.x] = xj[b];
            sy[threadIdx.x] = xj[b + 1];
            sz[threadIdx.x] = xj[b + 2];
            svx[threadIdx.x] = vj[b];
            svy[threadIdx.x] = vj[b + 1];
            svz[threadIdx.x] = vj[b + 2];
            sm[threadIdx.x] = mj[j];
        }
        __syncthreads();
        if (!valid) continue;
        for (int k = 0; k < cnt; ++k) {
            const int j = tb + k;
            if (j == self) continue;
            const double dx = sx[k] - x0, dy = sy[k] - y0, dz = sz[k] - z0;
            const double du = svx[k] - u0, dv = svy[k] - v0, dw = svz[k] - w0;
            const double r2n = dx * dx + dy * dy + dz * dz;
            const double rv = dx * du + dy * dv + dz * dw;
            const double rinv = rsqrt(r2n + eps2);
            const double r2inv = rinv * rinv;
            const double mr = sm[k] * rinv;
            const double mr3 = mr * r2inv;
            const double a3 = -3.0 * rv * r2inv;
            p -= mr;
            ax += mr3 * dx; ay += mr3 * dy; az += mr3 * dz;
            jx += mr3 * (du + a3 * dx); jy += mr3 * (dv + a3 * dy); jz += mr3 * (dw + a3 * dz);
            if (r2n < best) {
                best = r2n;
                bj = j;
            }
        }
    }
    if (!valid) return;
    if (nsplit == 1) {
        const size_t b = 3 * (size_t)i;
        acc[b] = ax; acc[b + 1] = ay; acc[b + 2] = az;
        jerk[b] = jx; jerk[b + 1] = jy; jerk[b + 2] = jz;
        pot[i] = p;
        nn[i] = bj < 0 ? 0 : bj;
        return;
    }
    NAPartial q;
    q.acc[0] = ax; q.acc[1] = ay; q.acc[2] = az;
    q.jerk[0] = jx; q.jerk[1] = jy; q.jerk[2] = jz;
    q.pot = p;
    q.nn_r2 = best;
    q.nn_j = bj;
    q.pad[0] = q.pad[1] = q.pad[2] = 0;
    scratch[(size_t)s * ni + i] = q;
}

// Adds the splits of every i in split order (deterministic).  Every record
// it reads was written by the force kernel of the same call, so the scratch
// needs no clearing between calls.
__global__ void noalloc_reduce_kernel(int ni, int nsplit, const NAPartial *__restrict__ scratch,
                                      double *__restrict__ acc, double *__restrict__ jerk,
                                      double *__restrict__ pot, int *__restrict__ nn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ni) return;
    NAPartial a = scratch[i];
    for (int s = 1; s < nsplit; ++s) {
        const NAPartial b = scratch[(size_t)s * ni + i];
        for (int c = 0; c < 3; ++c) {
            a.acc[c] += b.acc[c];
            a.jerk[c] += b.jerk[c];
        }
        a.pot += b.pot;
        na_take_min(a.nn_r2, a.nn_j, b.nn_r2, b.nn_j);
    }
    for (int c = 0; c < 3; ++c) {
        acc[3 * (size_t)i + c] = a.acc[c];
        jerk[3 * (size_t)i + c] = a.jerk[c];
    }
    pot[i] = a.pot;
    nn[i] = a.nn_j < 0 ? 0 : a.nn_j;
}

int fail(int code, const char *fmt, long long a = 0, long long b = 0) {
    char buf[256];
    snprintf(buf, sizeof buf, fmt, a, b);
    g6::record_error(buf);
    return code;
}

// Once per device, with that device current: look up the device address of
// the scratch array (host code may not use the symbol itself).
int setup_device(int dev, DeviceSetup **out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(-3, "g6b200_force_noalloc: device %lld out of range", dev);
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceSetup &d = g_setup[dev];
    if (!d.ready) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            return fail(-3, "g6b200_force_noalloc: cudaGetSymbolAddress failed (%lld: see cudaGetErrorString)",
                        (long long)e);
        }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return fail(-3, "g6b200_force_noalloc: cudaDeviceGetAttribute failed (%lld)", (long long)e);
        d.scratch = static_cast<NAPartial *>(p);
        d.num_sms = sms;
        d.ready = true;
    }
    *out = &d;
    return 0;
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" int g6b200_force_noalloc(int nj, const double *xj, const double *vj, const double *mj, int ni,
                                    const int *index_i, const double *xi, const double *vi, double eps2,
                                    double *acc, double *jerk, double *pot, int *nn, void *stream) {
    if (ni < 0 || nj < 0) return fail(-2, "g6b200_force_noalloc: negative size (ni=%lld, nj=%lld)", ni, nj);
    if (ni > kScratchRecords)
        return fail(-1, "g6b200_force_noalloc: ni=%lld exceeds the static scratch limit of %lld i-particles",
                    ni, kScratchRecords);
    if (ni == 0) return 0;
    if (!xi || !vi || !acc || !jerk || !pot || !nn || (nj > 0 && (!xj || !vj || !mj)))
        return fail(-2, "g6b200_force_noalloc: null buffer (ni=%lld, nj=%lld)", ni, nj);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(-3, "g6b200_force_noalloc: no current device");
    DeviceSetup *d = nullptr;
    int rc = setup_device(dev, &d);
    if (rc) return rc;
    // A CUDA error left pending by earlier work on this thread (the caller's
    // own or another library's) would be read back below as if this launch
    // had failed: report it as what it is and launch nothing.
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
        return fail(-3, "g6b200_force_noalloc: a CUDA error from earlier work was pending before this call "
                        "(%lld: see cudaGetErrorString); nothing launched", (long long)pending);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int iblocks = (ni + kTile - 1) / kTile;
    const int jtiles = nj > 0 ? (nj + kTile - 1) / kTile : 1;
    // Split j so that the grid covers the GPU twice, within the scratch.
    int nsplit = (2 * d->num_sms + iblocks - 1) / iblocks;
    nsplit = std::min(nsplit, kScratchRecords / ni);
    nsplit = std::min(nsplit, jtiles);
    nsplit = std::max(nsplit, 1);
    const int jper = ((jtiles + nsplit - 1) / nsplit) * kTile;
    nsplit = nj > 0 ? (nj + jper - 1) / jper : 1;
    noalloc_force_kernel<<<dim3(iblocks, nsplit), kTile, 0, st>>>(nj, xj, vj, mj, ni, index_i, xi, vi, eps2, jper,
                                                                  nsplit, d->scratch, acc, jerk, pot, nn);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(-3, "g6b200_force_noalloc: launch failed (%lld)", (long long)e);
    if (nsplit > 1) {
        noalloc_reduce_kernel<<<(ni + 255) / 256, 256, 0, st>>>(ni, nsplit, d->scratch, acc, jerk, pot, nn);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail(-3, "g6b200_force_noalloc: launch failed (%lld)", (long long)e);
    }
    return 0;
}
#pragma GCC visibility pop
