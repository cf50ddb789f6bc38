// f64 direct sum on the GPU: the accuracy reference of benchmarks at sampled targets.
// Restates fmm-ref/src/p2p.rs:147-186 (direct_sum): every pair with x != y exactly adds
// q / r and -q d / r^3 (r = sqrt(r2), r^3 = r2 * r, q d formed first), summed per
// target with Neumaier compensation; here the sources are split into chunks summed
// separately and the chunk sums are then added in chunk order with compensation.
// The result carries 1/(4 pi), like the FMM output.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fmm_b200.h"

namespace {

struct Neumaier {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double t) {
        double u = s + t;
        if (fabs(s) >= fabs(t)) c += (s - u) + t;
        else c += (t - u) + s;
        s = u;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

constexpr int kTile = 256;

__global__ void direct_partial_kernel(const double* __restrict__ src, const double* __restrict__ q, int64_t ns,
                                      const double* __restrict__ tgt, int64_t nt, int64_t chunk, int grad,
                                      double* __restrict__ part) {
    __shared__ double sx[kTile], sy[kTile], sz[kTile], sq[kTile];
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t c0 = blockIdx.y * chunk, c1 = c0 + chunk < ns ? c0 + chunk : ns;
    double x = 0, y = 0, z = 0;
    if (t < nt) {
        x = tgt[3 * t];
        y = tgt[3 * t + 1];
        z = tgt[3 * t + 2];
    }
    Neumaier ph, g0, g1, g2;
    for (int64_t b = c0; b < c1; b += kTile) {
        int cnt = (int)((c1 - b) < kTile ? (c1 - b) : kTile);
        __syncthreads();
        for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
            sx[j] = src[3 * (b + j)];
            sy[j] = src[3 * (b + j) + 1];
            sz[j] = src[3 * (b + j) + 2];
            sq[j] = q[b + j];
        }
        __syncthreads();
        if (t < nt)
            for (int j = 0; j < cnt; ++j) {
                if (x == sx[j] && y == sy[j] && z == sz[j]) continue;
                double d0 = __dsub_rn(x, sx[j]), d1 = __dsub_rn(y, sy[j]), d2 = __dsub_rn(z, sz[j]);
                double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
                double r = sqrt(r2);
                ph.add(sq[j] / r);
                if (grad) {
                    double r3 = __dmul_rn(r2, r);
                    g0.add(-(__dmul_rn(sq[j], d0) / r3));
                    g1.add(-(__dmul_rn(sq[j], d1) / r3));
                    g2.add(-(__dmul_rn(sq[j], d2) / r3));
                }
            }
    }
    if (t < nt) {
        double* o = part + ((int64_t)blockIdx.y * nt + t) * 4;
        o[0] = ph.value();
        o[1] = g0.value();
        o[2] = g1.value();
        o[3] = g2.value();
    }
}

__global__ void direct_combine_kernel(const double* __restrict__ part, int64_t nt, int nchunks, int grad,
                                      double* __restrict__ phi, double* __restrict__ g) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nt) return;
    Neumaier s[4];
    for (int c = 0; c < nchunks; ++c)
        for (int k = 0; k < 4; ++k) s[k].add(part[((int64_t)c * nt + t) * 4 + k]);
    const double f = 4.0 * 3.141592653589793;
    phi[t] = s[0].value() / f;
    if (grad)
        for (int k = 0; k < 3; ++k) g[3 * t + k] = s[k + 1].value() / f;
}

// Chunking of the sources shared by both entry points (same chunks, same bits).
int direct_chunks(size_t ns) { return ns > (1 << 16) ? 128 : 1; }

// Scratch of fmmgpu_direct_sum_noalloc: the per-chunk partial sums, nchunks x nt x 4
// doubles.  A module-scope array, so that the call allocates nothing; one per device.
__device__ __align__(256) double g_noalloc_part[FMMGPU_DIRECT_NOALLOC_SCRATCH_BYTES / sizeof(double)];

constexpr int kMaxDevices = 64;

}  // namespace

namespace fmmb {
void set_last_error(const std::string& message);  // evaluator.cu
}

extern "C" int fmmgpu_direct_sum(size_t ns, const double* src, const double* q, size_t nt, const double* tgt,
                                 double* phi, double* grad, int device) {
    auto fail = [](cudaError_t e) {
        fmmb::set_last_error(std::string("fmmgpu_direct_sum: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? FMMGPU_DEVICE_MEMORY : FMMGPU_DEVICE_ERROR;
    };
    if ((ns && (!src || !q)) || (nt && (!tgt || !phi))) {
        fmmb::set_last_error("fmmgpu_direct_sum: null buffer");
        return FMMGPU_INVALID_ARGUMENT;
    }
    if (nt == 0) return FMMGPU_OK;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e);
    const int nchunks = direct_chunks(ns);
    const int64_t chunk = ((int64_t)ns + nchunks - 1) / nchunks;
    double *dsrc = nullptr, *dq = nullptr, *dtgt = nullptr, *dpart = nullptr, *dphi = nullptr, *dg = nullptr;
    auto cleanup = [&] {
        cudaFree(dsrc);
        cudaFree(dq);
        cudaFree(dtgt);
        cudaFree(dpart);
        cudaFree(dphi);
        cudaFree(dg);
    };
    if ((e = cudaMalloc(&dsrc, 3 * ns * sizeof(double) + 8)) != cudaSuccess ||
        (e = cudaMalloc(&dq, ns * sizeof(double) + 8)) != cudaSuccess ||
        (e = cudaMalloc(&dtgt, 3 * nt * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&dpart, (size_t)nchunks * nt * 4 * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&dphi, nt * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&dg, 3 * nt * sizeof(double))) != cudaSuccess) {
        cleanup();
        return fail(e);
    }
    cudaMemcpy(dsrc, src, 3 * ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dq, q, ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dtgt, tgt, 3 * nt * sizeof(double), cudaMemcpyHostToDevice);
    dim3 grid((unsigned)((nt + 127) / 128), (unsigned)nchunks);
    direct_partial_kernel<<<grid, 128>>>(dsrc, dq, (int64_t)ns, dtgt, (int64_t)nt, chunk, grad != nullptr, dpart);
    direct_combine_kernel<<<(unsigned)((nt + 127) / 128), 128>>>(dpart, (int64_t)nt, nchunks, grad != nullptr, dphi, dg);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) {
        cudaMemcpy(phi, dphi, nt * sizeof(double), cudaMemcpyDeviceToHost);
        if (grad) cudaMemcpy(grad, dg, 3 * nt * sizeof(double), cudaMemcpyDeviceToHost);
    }
    cleanup();
    return e == cudaSuccess ? FMMGPU_OK : fail(e);
}

// Restores the calling thread's current device when a call returns.
struct CurrentDevice {
    int saved = -1;
    CurrentDevice() {
        if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
    }
    ~CurrentDevice() {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

// The same sums on device buffers with the scratch in g_noalloc_part: no device or host
// allocation, no synchronisation.  Its address on each device is looked up once, under a
// lock, by the first call there (the cached address assumes the device is not reset
// while the library is loaded).  Every scratch slot the combine reads is written by the
// partial kernel earlier in the same call, so nothing in it has to start at zero.  The
// calling thread's current device is the same on return as on entry.
extern "C" int fmmgpu_direct_sum_noalloc(size_t ns, const double* src, const double* q, size_t nt,
                                         const double* tgt, double* phi, double* grad, int device,
                                         void* stream) {
    if ((ns && (!src || !q)) || (nt && (!tgt || !phi))) {
        fmmb::set_last_error("fmmgpu_direct_sum_noalloc: null buffer");
        return FMMGPU_INVALID_ARGUMENT;
    }
    if (device < 0 || device >= kMaxDevices) {
        fmmb::set_last_error("fmmgpu_direct_sum_noalloc: device ordinal out of range");
        return FMMGPU_INVALID_ARGUMENT;
    }
    const int nchunks = direct_chunks(ns);
    const size_t capacity = FMMGPU_DIRECT_NOALLOC_SCRATCH_BYTES / (4 * sizeof(double));  // (chunk, target) slots
    if (nt > capacity / (size_t)nchunks) {
        fmmb::set_last_error("fmmgpu_direct_sum_noalloc: " + std::to_string(nt) + " targets x " +
                             std::to_string(nchunks) + " source chunks need " +
                             std::to_string((unsigned long long)nt * nchunks * 4 * sizeof(double)) +
                             " bytes of scratch; the static scratch holds " +
                             std::to_string((unsigned long long)FMMGPU_DIRECT_NOALLOC_SCRATCH_BYTES) +
                             " bytes (at most " + std::to_string(capacity / nchunks) + " targets here)");
        return FMMGPU_INVALID_ARGUMENT;
    }
    if (nt == 0) return FMMGPU_OK;
    auto fail = [](const char* what, cudaError_t e) {
        fmmb::set_last_error(std::string("fmmgpu_direct_sum_noalloc: ") + what + ": " + cudaGetErrorString(e));
        return FMMGPU_DEVICE_ERROR;
    };
    CurrentDevice keep;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail("cudaSetDevice", e);
    // an error left by earlier work on this thread is reported as such, not cleared, and
    // nothing is launched
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) return fail("a CUDA error from before this call is pending", e);
    static std::mutex mu;
    static double* scratch[kMaxDevices] = {};
    double* part;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!scratch[device]) {
            void* addr = nullptr;
            e = cudaGetSymbolAddress(&addr, g_noalloc_part);
            if (e != cudaSuccess) return fail("cudaGetSymbolAddress", e);
            scratch[device] = static_cast<double*>(addr);
        }
        part = scratch[device];
    }
    const int64_t chunk = ((int64_t)ns + nchunks - 1) / nchunks;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    dim3 grid((unsigned)((nt + 127) / 128), (unsigned)nchunks);
    direct_partial_kernel<<<grid, 128, 0, s>>>(src, q, (int64_t)ns, tgt, (int64_t)nt, chunk, grad != nullptr, part);
    direct_combine_kernel<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(part, (int64_t)nt, nchunks, grad != nullptr,
                                                                       phi, grad);
    e = cudaGetLastError();
    return e == cudaSuccess ? FMMGPU_OK : fail("launch", e);
}

// ---- Helmholtz: e^{ikr}/(4 pi r), the terms of fmm-ref/src/helmholtz/p2p.rs:315-375
// (direct_sum: Neumaier per real component, coincident pairs skipped) ----
namespace {

__global__ void helm_direct_kernel(double kre, double kim, const double* __restrict__ src,
                                   const double* __restrict__ q, int64_t ns, const double* __restrict__ tgt,
                                   int64_t nt, int grad, double* __restrict__ phi, double* __restrict__ g) {
    __shared__ double sx[kTile], sy[kTile], sz[kTile], sqr[kTile], sqi[kTile];
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double x = 0, y = 0, z = 0;
    if (t < nt) {
        x = tgt[3 * t];
        y = tgt[3 * t + 1];
        z = tgt[3 * t + 2];
    }
    Neumaier s[8];
    for (int64_t b = 0; b < ns; b += kTile) {
        const int cnt = (int)((ns - b) < kTile ? (ns - b) : kTile);
        __syncthreads();
        for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
            sx[j] = src[3 * (b + j)];
            sy[j] = src[3 * (b + j) + 1];
            sz[j] = src[3 * (b + j) + 2];
            sqr[j] = q[2 * (b + j)];
            sqi[j] = q[2 * (b + j) + 1];
        }
        __syncthreads();
        if (t < nt)
            for (int j = 0; j < cnt; ++j) {
                if (x == sx[j] && y == sy[j] && z == sz[j]) continue;
                const double d0 = __dsub_rn(x, sx[j]), d1 = __dsub_rn(y, sy[j]), d2 = __dsub_rn(z, sz[j]);
                const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2));
                const double r = sqrt(r2);
                const double damping = -(kim * r), phase = kre * r;
                double sn, cs;
                sincos(phase, &sn, &cs);
                const double decay = exp(damping);
                const double er = decay * cs, ei = decay * sn;
                const double qer = __dsub_rn(__dmul_rn(sqr[j], er), __dmul_rn(sqi[j], ei));
                const double qei = __dadd_rn(__dmul_rn(sqr[j], ei), __dmul_rn(sqi[j], er));
                s[0].add(qer / r);
                s[1].add(qei / r);
                if (grad) {
                    const double r3 = __dmul_rn(r2, r);
                    const double fr = damping - 1.0, fi = phase;
                    const double fer = __dsub_rn(__dmul_rn(fr, er), __dmul_rn(fi, ei));
                    const double fei = __dadd_rn(__dmul_rn(fr, ei), __dmul_rn(fi, er));
                    const double gr = fer / r3, gi = fei / r3;
                    const double qgr = __dsub_rn(__dmul_rn(sqr[j], gr), __dmul_rn(sqi[j], gi));
                    const double qgi = __dadd_rn(__dmul_rn(sqr[j], gi), __dmul_rn(sqi[j], gr));
                    const double dd[3] = {d0, d1, d2};
                    for (int k = 0; k < 3; ++k) {
                        s[2 + 2 * k].add(__dmul_rn(qgr, dd[k]));
                        s[3 + 2 * k].add(__dmul_rn(qgi, dd[k]));
                    }
                }
            }
    }
    if (t < nt) {
        const double f = 4.0 * 3.141592653589793;
        phi[2 * t] = s[0].value() / f;
        phi[2 * t + 1] = s[1].value() / f;
        if (grad)
            for (int k = 0; k < 6; ++k) g[6 * t + k] = s[2 + k].value() / f;
    }
}

}  // namespace

extern "C" int fmmgpu_helmholtz_direct_sum(double kre, double kim, size_t ns, const double* src, const double* q,
                                           size_t nt, const double* tgt, double* phi, double* grad, int device) {
    auto fail = [](cudaError_t e) {
        fmmb::set_last_error(std::string("fmmgpu_helmholtz_direct_sum: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? FMMGPU_DEVICE_MEMORY : FMMGPU_DEVICE_ERROR;
    };
    if ((ns && (!src || !q)) || (nt && (!tgt || !phi))) {
        fmmb::set_last_error("fmmgpu_helmholtz_direct_sum: null buffer");
        return FMMGPU_INVALID_ARGUMENT;
    }
    if (!std::isfinite(kre) || !std::isfinite(kim)) {
        fmmb::set_last_error("fmmgpu_helmholtz_direct_sum: the wavenumber must be finite");
        return FMMGPU_INVALID_ARGUMENT;
    }
    if (nt == 0) return FMMGPU_OK;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e);
    double *dsrc = nullptr, *dq = nullptr, *dtgt = nullptr, *dphi = nullptr, *dg = nullptr;
    auto cleanup = [&] {
        cudaFree(dsrc);
        cudaFree(dq);
        cudaFree(dtgt);
        cudaFree(dphi);
        cudaFree(dg);
    };
    if ((e = cudaMalloc(&dsrc, 3 * ns * sizeof(double) + 8)) != cudaSuccess ||
        (e = cudaMalloc(&dq, 2 * ns * sizeof(double) + 8)) != cudaSuccess ||
        (e = cudaMalloc(&dtgt, 3 * nt * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&dphi, 2 * nt * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&dg, 6 * nt * sizeof(double))) != cudaSuccess) {
        cleanup();
        return fail(e);
    }
    cudaMemcpy(dsrc, src, 3 * ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dq, q, 2 * ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dtgt, tgt, 3 * nt * sizeof(double), cudaMemcpyHostToDevice);
    helm_direct_kernel<<<(unsigned)((nt + 127) / 128), 128>>>(kre, kim, dsrc, dq, (int64_t)ns, dtgt, (int64_t)nt,
                                                            grad != nullptr, dphi, dg);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) {
        cudaMemcpy(phi, dphi, 2 * nt * sizeof(double), cudaMemcpyDeviceToHost);
        if (grad) cudaMemcpy(grad, dg, 6 * nt * sizeof(double), cudaMemcpyDeviceToHost);
    }
    cleanup();
    return e == cudaSuccess ? FMMGPU_OK : fail(e);
}
