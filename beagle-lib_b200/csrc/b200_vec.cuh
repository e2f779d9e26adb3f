// Four-state vector loads and stores: one pattern-category row of the
// [pattern][category][state] partials layout is 16 bytes (FP32) or 32 bytes
// (FP64).  ld4 is a plain load (data written earlier in the same launch);
// ldg4 goes through the read-only path (matrices, never written by the kernel).
#pragma once
#include <cuda_runtime.h>

namespace b200 {

__device__ __forceinline__ void ld4(const float* p, float v[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ldg4(const float* p, float v[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ldg4(const double* p, double v[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const float v[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double v[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// 1 / x correctly rounded (the IEEE quotient of 1 by x, the value `1 / x`
// gives), through the reciprocal intrinsics instead of a division.
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }

// Natural log of a positive rescaling factor, in FP64.  FP64 partials: log.
// FP32 partials: m = 2^e f with f in [1, 2), log m = (e + log2 f) ln 2 with the
// integer part exact and log2 f from the hardware base-2 logarithm (__log2f,
// absolute error below 2^-22 on [0.5, 2]): below 2e-7 whatever the exponent,
// the accuracy the FP32 partials carry already.
__device__ __forceinline__ double scale_log(double m) { return log(m); }
__device__ __forceinline__ double scale_log(float m) {
    const int bits = __float_as_int(m);
    const int ex = (bits >> 23) & 0xff;
    if (ex == 0 || ex == 0xff) return log((double)m);   // subnormal, infinite, NaN
    const float f = __int_as_float((bits & 0x007fffff) | 0x3f800000);
    constexpr double kLn2 = 0.69314718055994530942;
    return ((double)(ex - 127) + (double)__log2f(f)) * kLn2;
}

}  // namespace b200
