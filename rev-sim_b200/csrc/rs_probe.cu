// rs_probe.cu -- measured FP32 FMA throughput of the current GPU, the roofline
// denominator for the FP32-pipe-bound step kernels (their work is scalar FP32
// arithmetic on CUDA cores, not tensor-core or HBM bound).
#include <cuda_runtime.h>

#include "revsim.h"

namespace {

constexpr int kChains = 16;
constexpr int kIters = 2048;

__global__ void __launch_bounds__(256) k_ffma(float *out, float a, float b) {
    float acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) acc[c] = threadIdx.x * 1e-3f + c;
    for (int it = 0; it < kIters; it++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) acc[c] = __fmaf_rn(acc[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += acc[c];
    if (s == 12345.678f) out[blockIdx.x] = s;   // keeps the chains live
}

}  // namespace

extern "C" int32_t revsim_probe_fp32_tflops(int32_t device, double *tflops) {
    if (!tflops) return REVSIM_ERR_BADARG;
    if (cudaSetDevice(device) != cudaSuccess) return REVSIM_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256;
    float *out = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMalloc(&out, sizeof(float) * blocks) != cudaSuccess) return REVSIM_ERR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int w = 0; w < 3; w++) k_ffma<<<blocks, threads>>>(out, 0.999f, 1e-4f);
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0);
        k_ffma<<<blocks, threads>>>(out, 0.999f, 1e-4f);
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
