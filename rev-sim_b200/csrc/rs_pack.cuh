// rs_pack.cuh -- two neighbour entries per lane in one register pair (sm_100a).
//
// The FP32 step kernels evaluate the pair terms of two neighbour-row entries at once: the .x
// half of every value belongs to one entry, the .y half to the other.  Products, sums and
// fused multiply-adds are the packed sm_100 instructions (__fadd2_rn, __fmul2_rn, __ffma2_rn:
// one instruction for both halves, each half rounded exactly as __fadd_rn, __fmul_rn,
// __fmaf_rn), which halves the FP32 instructions a row costs.  Square roots, exponentials and
// comparisons are per half.
#pragma once

#include <cuda_runtime.h>

#include "rs_device.cuh"

namespace rs {

template <typename R> struct PkT;
template <> struct PkT<float> { using T = float2; };
template <> struct PkT<double> { using T = double2; };

__device__ __forceinline__ float2 pk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 pk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 pk1(float a) { return make_float2(a, a); }
__device__ __forceinline__ double2 pk1(double a) { return make_double2(a, a); }

// a - b as fma(b, -1, a): b * -1 is exact, so the one rounding gives the bits of
// __fsub_rn(a, b).
__device__ __forceinline__ float2 xadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 xmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 xfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 xsub(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
__device__ __forceinline__ float2 xneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 xrsqrt(float2 a) { return make_float2(xrsqrt(a.x), xrsqrt(a.y)); }

// FP64 (no packed form): per half, for code written once for both precisions.
__device__ __forceinline__ double2 xadd(double2 a, double2 b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 xmul(double2 a, double2 b) {
    return make_double2(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
}
__device__ __forceinline__ double2 xfma(double2 a, double2 b, double2 c) {
    return make_double2(__fma_rn(a.x, b.x, c.x), __fma_rn(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 xsub(double2 a, double2 b) {
    return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
__device__ __forceinline__ double2 xneg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double2 xrsqrt(double2 a) { return make_double2(xrsqrt(a.x), xrsqrt(a.y)); }

}  // namespace rs
