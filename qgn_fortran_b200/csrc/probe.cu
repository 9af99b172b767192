// probe.cu -- FP64 FMA throughput probe (the denominator of the transforms' FLOP fraction).
#include <cuda_runtime.h>

#include "../../include/qgn_gpu.h"
#include "../../include/qgn_probe.h"
#include "launch.cuh"

namespace {

constexpr int kChains = 32;      // independent FMA chains per thread
constexpr int kThreads = 256;
constexpr int kCtasPerSm = 8;
constexpr int kIters = 2048;     // iterations of kChains FMAs: ~40 GFLOP per launch on 148 SMs

// a <- a*b + c on kChains registers; b and c are launch arguments, so nothing folds, and every
// thread stores its sum, so no chain is dead.  With b < 1 the chains converge to c/(1-b).
__global__ void __launch_bounds__(kThreads) k_fp64_fma(double* __restrict__ out, int iters, double b, double c) {
    QGN_PDL_ENTRY();
    double a[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = 1.0e-3 * threadIdx.x + i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < kChains; ++i) a[i] = fma(a[i], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < kChains; ++i) s += a[i];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

struct Cleanup {
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double* out = nullptr;
    ~Cleanup() {
        if (st) cudaStreamSynchronize(st);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (out) cudaFree(out);
        if (st) cudaStreamDestroy(st);
    }
};

}  // namespace

extern "C" int qgn_probe_fp64_fma(int reps, double* tflops, double* ms) {
    if (!tflops) return QGN_ERR_ARG;
    if (reps <= 0) reps = 5;
    int dev = 0, nsm = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return QGN_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major != 10)
        return QGN_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return QGN_ERR_CUDA;
    const int grid = nsm * kCtasPerSm;
    Cleanup c;
    if (cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking) != cudaSuccess) return QGN_ERR_CUDA;
    if (cudaEventCreate(&c.e0) != cudaSuccess || cudaEventCreate(&c.e1) != cudaSuccess) return QGN_ERR_CUDA;
    if (cudaMalloc(&c.out, sizeof(double) * (size_t)grid * kThreads) != cudaSuccess) return QGN_ERR_CUDA;
    const double b = 0.9999999, cc = 1.0e-7;
    float best = -1.0f;
    for (int r = 0; r < reps + 2; ++r) {
        if (cudaEventRecord(c.e0, c.st) != cudaSuccess) return QGN_ERR_CUDA;
        if (::qgn::launch(k_fp64_fma, grid, kThreads, 0, c.st, c.out, kIters, b, cc) != cudaSuccess) return QGN_ERR_CUDA;
        if (cudaEventRecord(c.e1, c.st) != cudaSuccess) return QGN_ERR_CUDA;
        if (cudaEventSynchronize(c.e1) != cudaSuccess) return QGN_ERR_CUDA;
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, c.e0, c.e1) != cudaSuccess) return QGN_ERR_CUDA;
        if (r >= 2 && (best < 0.0f || t < best)) best = t;
    }
    const double flops = 2.0 * kChains * (double)kIters * grid * kThreads;
    *tflops = flops / (best * 1.0e-3) / 1.0e12;
    if (ms) *ms = best;
    return QGN_OK;
}
