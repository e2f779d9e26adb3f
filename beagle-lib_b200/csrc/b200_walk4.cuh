// Device code shared by the S = 4 partials kernels of one instance
// (k_partials.cu) and of a batch of instances (k_batch.cu): the per-op body of
// the post- and pre-order walks with their fused rescaling.  The arithmetic
// is described in k_partials.cu.
#pragma once
#include "b200_kernels.h"
#include "b200_vec.cuh"

namespace b200 {
namespace {

// Store the scale factor of one pattern (see the file comment): its log
// (scale_log) stored and accumulated in FP64, into the cumulative buffer
// `cum` and/or the caller's register `acc` when given.
template <typename Real>
__device__ __forceinline__ void store_scale(Real m, double* scale_write, double* cum, int p,
                                            int log_scalers, double* acc = nullptr) {
    const double lm = scale_log(m);
    scale_write[p] = log_scalers ? lm : (double)m;
    if (cum) cum[p] += lm;
    if (acc) *acc += lm;
}

// ------------------------------------------------------------ S = 4 kernels
// One thread per (pattern, category): a category's four states are one
// 16-byte (FP32) / 32-byte (FP64) vector, so consecutive threads read and
// write consecutive vectors of the [pattern][category][state] layout.  The C
// threads of a pattern form an aligned lane group; the rescaling maximum over
// categories is a shuffle reduction inside that group.  Each thread carries
// PPT patterns (PPT chosen at launch so the grid is a single resident wave),
// and the op descriptors are staged in shared memory chunk by chunk so the
// per-op loads (children, matrices) all issue together.
constexpr int kOpChunk = 64;
constexpr int kT4 = 256;        // threads per CTA of the S = 4 kernels

__device__ __forceinline__ void stage_ops(OpDesc* s_ops, const OpDesc* __restrict__ ops, int n) {
    const int* src = reinterpret_cast<const int*>(ops);
    int* dst = reinterpret_cast<int*>(s_ops);
    const int words = n * (int)(sizeof(OpDesc) / sizeof(int));
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
}

// y[i] = (M_c . x)[i] for one operand of one category: partials vector x, or
// column s of M_c (pad value for the missing state).
template <typename Real>
__device__ __forceinline__ void operand4c(const Real* __restrict__ Mc, bool states, int s,
                                          const Real x[4], Real pad, Real y[4]) {
    if (states) {
#pragma unroll
        for (int i = 0; i < 4; ++i) y[i] = (s < 4) ? __ldg(Mc + i * 4 + (s & 3)) : pad;
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Real m[4];
            ldg4(Mc + i * 4, m);
            y[i] = m[0] * x[0] + m[1] * x[1] + m[2] * x[2] + m[3] * x[3];
        }
    }
}

template <int C, typename Real>
__device__ __forceinline__ Real group_max(Real v) {
#pragma unroll
    for (int o = 1; o < C; o <<= 1) {
        const Real u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u > v ? u : v;
    }
    return v;
}

// Rescale / fixed-scale and store one pattern-category vector.
// RANGED: the list has partition ops (own pattern range and cumulative
// buffer); whole-instance lists skip those checks.
template <typename Real, int C, bool RANGED = true>
__device__ __forceinline__ void finish4c(const OpDesc& op, Real out[4], int p, bool valid, int c,
                                         double* cum, int log_scalers, double* acc = nullptr) {
    if (RANGED) {
        valid = valid && p >= op.p_begin && p < op.p_end;
        if (op.cum) cum = op.cum;
    }
    if (op.scale_write) {
        Real m = out[0];
#pragma unroll
        for (int i = 1; i < 4; ++i) m = out[i] > m ? out[i] : m;
        m = group_max<C>(m);
        if (m == Real(0)) m = Real(1);
        const Real inv = recip(m);
#pragma unroll
        for (int i = 0; i < 4; ++i) out[i] *= inv;
        if (valid && c == 0) store_scale(m, op.scale_write, cum, p, log_scalers, acc);
    } else if (op.scale_read) {
        const Real inv = recip((Real)op.scale_read[p]);
#pragma unroll
        for (int i = 0; i < 4; ++i) out[i] *= inv;
    }
    if (valid) st4(static_cast<Real*>(op.dest) + ((size_t)p * C + c) * 4, out);
}

// One post-order op for this thread's PPT patterns (p0 + k pstride).
// acc (PPT = 1): a register that also receives this pattern's log scale
// factor (lane c == 0).
template <typename Real, int C, int PPT, bool RANGED>
__device__ __forceinline__ void post4_op(const OpDesc& op, int c, int p0, int pstride, int Pp,
                                         double* cum, int log_scalers, double* acc = nullptr) {
    const bool st1 = op.kind & kX1States, st2 = op.kind & kX2States;
    const Real* M1 = static_cast<const Real*>(op.m1) + c * 16;
    const Real* M2 = static_cast<const Real*>(op.m2) + c * 16;
    Real x1[PPT][4], x2[PPT][4];
    int s1[PPT], s2[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int p = min(p0 + k * pstride, Pp - 1);
        if (st1) s1[k] = static_cast<const int*>(op.x1)[p];
        else ld4(static_cast<const Real*>(op.x1) + ((size_t)p * C + c) * 4, x1[k]);
        if (st2) s2[k] = static_cast<const int*>(op.x2)[p];
        else ld4(static_cast<const Real*>(op.x2) + ((size_t)p * C + c) * 4, x2[k]);
    }
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int p = p0 + k * pstride;
        Real y1[4], y2[4];
        operand4c(M1, st1, s1[k], x1[k], (Real)op.pad1, y1);
        operand4c(M2, st2, s2[k], x2[k], (Real)op.pad2, y2);
#pragma unroll
        for (int i = 0; i < 4; ++i) y1[i] *= y2[i];
        finish4c<Real, C, RANGED>(op, y1, min(p, Pp - 1), p < Pp, c, cum, log_scalers, acc);
    }
}

// One pre-order op for this thread's PPT patterns.
template <typename Real, int C, int PPT, bool RANGED>
__device__ __forceinline__ void pre4_op(const OpDesc& op, int c, int p0, int pstride, int Pp,
                                        int log_scalers) {
    const bool st2 = op.kind & kX2States;
    const bool tr = op.kind & kM1Transposed;
    const Real* M1 = static_cast<const Real*>(op.m1) + c * 16;
    const Real* M2 = static_cast<const Real*>(op.m2) + c * 16;
    Real pv[PPT][4], x2[PPT][4];
    int s2[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int p = min(p0 + k * pstride, Pp - 1);
        ld4(static_cast<const Real*>(op.x1) + ((size_t)p * C + c) * 4, pv[k]);
        if (st2) s2[k] = static_cast<const int*>(op.x2)[p];
        else ld4(static_cast<const Real*>(op.x2) + ((size_t)p * C + c) * 4, x2[k]);
    }
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int p = p0 + k * pstride;
        Real z[4];
        operand4c(M2, st2, s2[k], x2[k], (Real)op.pad2, z);
#pragma unroll
        for (int i = 0; i < 4; ++i) z[i] *= pv[k][i];
        Real out[4] = {0, 0, 0, 0};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Real m[4];
            if (tr) {
#pragma unroll
                for (int j = 0; j < 4; ++j) m[j] = __ldg(M1 + j * 4 + i);
            } else {
                ldg4(M1 + i * 4, m);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) out[j] += m[j] * z[i];
        }
        finish4c<Real, C, RANGED>(op, out, min(p, Pp - 1), p < Pp, c, nullptr, log_scalers);
    }
}

}  // namespace
}  // namespace b200
