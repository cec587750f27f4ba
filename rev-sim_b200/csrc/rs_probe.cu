// rs_probe.cu -- measured FP32 and FP64 FMA throughput of the current GPU, the roofline
// denominators for the FP32-pipe-bound step kernels of the mixed-precision water engine and
// the FP64 kernels of the gas-in-water engine (scalar arithmetic on CUDA cores, not tensor-
// core or HBM bound).
#include <cuda_runtime.h>

#include "revsim.h"

namespace {

constexpr int kChains = 16;
constexpr int kIters = 2048;

__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T>
__global__ void __launch_bounds__(256) k_fma(T *out, T a, T b) {
    T acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) acc[c] = threadIdx.x * T(1e-3) + c;
    for (int it = 0; it < kIters; it++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) acc[c] = fma_t(acc[c], a, b);
    }
    T s = T(0);
#pragma unroll
    for (int c = 0; c < kChains; c++) s += acc[c];
    if (s == T(12345.678)) out[blockIdx.x] = s;   // keeps the chains live
}

template <typename T>
int32_t probe(int32_t device, double *tflops) {
    if (!tflops) return REVSIM_ERR_BADARG;
    if (cudaSetDevice(device) != cudaSuccess) return REVSIM_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256;
    T *out = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMalloc(&out, sizeof(T) * blocks) != cudaSuccess) return REVSIM_ERR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int w = 0; w < 3; w++) k_fma<T><<<blocks, threads>>>(out, T(0.999), T(1e-4));
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0);
        k_fma<T><<<blocks, threads>>>(out, T(0.999), T(1e-4));
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return REVSIM_ERR_CUDA;
    const double flops = 2.0 * kChains * kIters * (double)blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return REVSIM_OK;
}

}  // namespace

extern "C" int32_t revsim_probe_fp32_tflops(int32_t device, double *tflops) {
    return probe<float>(device, tflops);
}

extern "C" int32_t revsim_probe_fp64_tflops(int32_t device, double *tflops) {
    return probe<double>(device, tflops);
}
