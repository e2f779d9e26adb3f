// Post-order and pre-order partials: one launch walks a whole operation list.
//
// Patterns are independent given the tree and the model, so the launch is
// split over pattern tiles only and every CTA walks the full op list for its
// own patterns: an op's children were produced earlier in the same CTA, and no
// grid-wide synchronisation is needed between dependent ops.
//
// Per operation (CPU/BeagleCPUImpl.hpp:1497-1686, :4226-4524, :4665-4722):
//   post:  dest[c,p,i] = (sum_j M1[c][i][j] x1[c,p,j]) * (sum_j M2[c][i][j] x2[c,p,j])
//          a compact tip operand selects column x[p] of M (the missing state
//          selects the matrix's pad value);
//   pre:   dest[c,p,j] = sum_i M1[c][i][j] * x1[c,p,i] * (M2 . x2)[c,p,i]
//          (CPU/BeagleCPUImpl.hpp:4530-4662; M1 given transposed when the
//          op carries kM1Transposed);
//   rescale (CPU/BeagleCPUImpl.hpp:4008-4056): m[p] = max_{c,i} dest (0 -> 1),
//          dest *= 1/m, scale[p] = log m (LOG scalers) or m (RAW), and
//          cumulative[p] += log m when a cumulative buffer is given;
//   fixed scaling: dest *= 1/scale_read[p].
//
// This file holds the S = 4 kernels: one thread per (pattern, category),
// vector loads and stores of one 4-state row, lane-group shuffles for the
// rescaling maximum.  HBM-bound.  Other state counts: k_generic.cu.
#include <algorithm>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "b200_kernels.h"
#include "b200_vec.cuh"
#include "b200_walk4.cuh"

namespace b200 {

namespace {

template <typename Real, int C, int PPT, bool RANGED, int MINB = 1>
__global__ void __launch_bounds__(kT4, MINB)
k_post4(const OpDesc* __restrict__ ops, int nops, int Pp, double* cum, int log_scalers) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    OpDesc* s_ops = reinterpret_cast<OpDesc*>(smem_raw);
    const int c = threadIdx.x % C;
    const int ppb = kT4 / C;                                 // patterns per CTA per slot
    const int pstride = gridDim.x * ppb;
    const int p0 = blockIdx.x * ppb + threadIdx.x / C;
    for (int o0 = 0; o0 < nops; o0 += kOpChunk) {
        const int n = min(kOpChunk, nops - o0);
        __syncthreads();
        stage_ops(s_ops, ops + o0, n);
        __syncthreads();
        for (int oi = 0; oi < n; ++oi)
            post4_op<Real, C, PPT, RANGED>(s_ops[oi], c, p0, pstride, Pp, cum, log_scalers);
    }
}

template <typename Real, int C, int PPT, bool RANGED, int MINB = 1>
__global__ void __launch_bounds__(kT4, MINB)
k_pre4(const OpDesc* __restrict__ ops, int nops, int Pp, int log_scalers) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    OpDesc* s_ops = reinterpret_cast<OpDesc*>(smem_raw);
    const int c = threadIdx.x % C;
    const int ppb = kT4 / C;
    const int pstride = gridDim.x * ppb;
    const int p0 = blockIdx.x * ppb + threadIdx.x / C;
    for (int o0 = 0; o0 < nops; o0 += kOpChunk) {
        const int n = min(kOpChunk, nops - o0);
        __syncthreads();
        stage_ops(s_ops, ops + o0, n);
        __syncthreads();
        for (int oi = 0; oi < n; ++oi)
            pre4_op<Real, C, PPT, RANGED>(s_ops[oi], c, p0, pstride, Pp, log_scalers);
    }
}

// The same walks with the op list passed by value as a kernel parameter (at
// most kParamOps ops a launch, CUDA 12.1+ on sm_70+; longer lists run as
// consecutive launches, run_param4): descriptor fields are then warp-uniform
// constant-bank reads instead of shared-memory loads, and no staging or
// barriers are needed between ops.
constexpr int kParamOps = 256;
struct OpParams {
    OpDesc op[kParamOps];
};

template <typename Real, int C, int PPT, bool RANGED>
__global__ void __launch_bounds__(kT4)
k_post4c(const __grid_constant__ OpParams P, int nops, int Pp, double* cum, int log_scalers) {
    const int c = threadIdx.x % C;
    const int ppb = kT4 / C;
    const int pstride = gridDim.x * ppb;
    const int p0 = blockIdx.x * ppb + threadIdx.x / C;
    for (int o = 0; o < nops; ++o)
        post4_op<Real, C, PPT, RANGED>(P.op[o], c, p0, pstride, Pp, cum, log_scalers);
}

template <typename Real, int C, int PPT, bool RANGED>
__global__ void __launch_bounds__(kT4)
k_pre4c(const __grid_constant__ OpParams P, int nops, int Pp, int log_scalers) {
    const int c = threadIdx.x % C;
    const int ppb = kT4 / C;
    const int pstride = gridDim.x * ppb;
    const int p0 = blockIdx.x * ppb + threadIdx.x / C;
    for (int o = 0; o < nops; ++o)
        pre4_op<Real, C, PPT, RANGED>(P.op[o], c, p0, pstride, Pp, log_scalers);
}

// The parameter-list post-order walk with the scale accumulation and the
// root log-likelihood fused (beagleB200UpdatePartialsWithRootLogLikelihood):
// each thread keeps its pattern's sum of log scale factors in a register
// (CPU/BeagleCPUImpl.hpp:2763-2801, as resetScaleFactors + accumulateScale-
// Factors over the list's scale buffers), re-reads the root row it wrote in
// the last op, and forms the site lnL of CPU/BeagleCPUImpl.hpp:2630-2691:
// log sum_c w_c sum_i pi_i root[c][i] + cumulative, the category sum by
// shuffles inside the pattern's lane group.  Per-warp weighted sums go to
// `block` for the final fixed-order sum.
// Matrices of a chunk of root_chunk ops (16 KB) in shared memory,
// [op][M1, M2][c][row] rows of 4 values.  The row order inside a category's block is rotated by
// c / 2 so the C lane-group members reading row i of their own category hit
// distinct banks (FP32: C 16-byte pieces in one wavefront).
template <typename Real, int C>
constexpr int root_chunk() {
    return 16384 / (2 * C * 16 * (int)sizeof(Real)) < 64 ? 16384 / (2 * C * 16 * (int)sizeof(Real))
                                                         : 64;
}

template <typename Real, int C>
__device__ __forceinline__ int mat_row(int k, int w, int c, int i) {
    return (((k * 2 + w) * C + c) * 4 + ((i + (c >> 1)) & 3)) * 4;
}

// An operand given as tip states reads one column of M_c, so its matrix is
// staged transposed: that column is then one row of 4 values.
// PRE (pre-order ops): the first matrix is P of the op's branch, applied as
// out_j = sum_i P[i][j] z_i, so it is staged as rows of P (given transposed,
// kM1Transposed, it is turned back); the second is the sibling's, as for a
// post-order child.
template <typename Real, int C, bool PRE = false>
__device__ __forceinline__ void stage_mats(Real* sm, const OpDesc* ops, int n) {
    for (int u = threadIdx.x; u < n * 2 * C * 4; u += kT4) {
        const int i = u & 3, c = (u >> 2) % C, w = (u / (4 * C)) & 1, k = u / (8 * C);
        const OpDesc& op = ops[k];
        const Real* M = static_cast<const Real*>(w ? op.m2 : op.m1) + c * 16;
        const bool tr = w ? (op.kind & kX2States) != 0
                          : (op.kind & (PRE ? kM1Transposed : kX1States)) != 0;
        Real v[4];
        if (tr) {
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = __ldg(M + j * 4 + i);
        } else {
            ldg4(M + i * 4, v);
        }
        Real* d = sm + mat_row<Real, C>(k, w, c, i);
#pragma unroll
        for (int j = 0; j < 4; ++j) d[j] = v[j];
    }
}

template <typename Real>
__device__ __forceinline__ void lds4(const Real* r, Real m[4]) {
    if constexpr (sizeof(Real) == 4) {
        const float4 q = *reinterpret_cast<const float4*>(r);
        m[0] = q.x; m[1] = q.y; m[2] = q.z; m[3] = q.w;
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) m[j] = r[j];
    }
}

// y = M_c . x (or column s of M_c, a row of the transposed image) with the
// rows from the staged chunk.
template <typename Real, int C>
__device__ __forceinline__ void operand4s(const Real* sm, int k, int w, int c, bool states, int s,
                                          const Real x[4], Real pad, Real y[4]) {
    if (states) {
        lds4(sm + mat_row<Real, C>(k, w, c, s & 3), y);
#pragma unroll
        for (int i = 0; i < 4; ++i) y[i] = s < 4 ? y[i] : pad;
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Real m[4];
            lds4(sm + mat_row<Real, C>(k, w, c, i), m);
            y[i] = m[0] * x[0] + m[1] * x[1] + m[2] * x[2] + m[3] * x[3];
        }
    }
}

template <typename Real, int C>
__global__ void __launch_bounds__(kT4, sizeof(Real) == 4 ? 6 : 1)
k_post4root(const __grid_constant__ OpParams P, int nops, int Pp, int Pn, double* cum,
            int log_scalers, const double* __restrict__ catw, const double* __restrict__ freqs,
            const double* __restrict__ patw, double* site, double* block) {
    constexpr int K = root_chunk<Real, C>();
    __shared__ __align__(16) Real s_m[K * 2 * C * 16];
    const int c = threadIdx.x % C;
    const int p0 = blockIdx.x * (kT4 / C) + threadIdx.x / C;
    const int p = min(p0, Pp - 1);
    const bool valid = p0 < Pp;
    double acc = 0;
    for (int o0 = 0; o0 < nops; o0 += K) {
        const int n = min(K, nops - o0);
        __syncthreads();
        stage_mats<Real, C>(s_m, P.op + o0, n);
        __syncthreads();
        for (int k = 0; k < n; ++k) {
            const OpDesc& op = P.op[o0 + k];
            const bool st1 = op.kind & kX1States, st2 = op.kind & kX2States;
            Real x1[4], x2[4];
            int s1 = 0, s2 = 0;
            if (st1) s1 = static_cast<const int*>(op.x1)[p];
            else ld4(static_cast<const Real*>(op.x1) + ((size_t)p * C + c) * 4, x1);
            if (st2) s2 = static_cast<const int*>(op.x2)[p];
            else ld4(static_cast<const Real*>(op.x2) + ((size_t)p * C + c) * 4, x2);
            Real y1[4], y2[4];
            operand4s<Real, C>(s_m, k, 0, c, st1, s1, x1, (Real)op.pad1, y1);
            operand4s<Real, C>(s_m, k, 1, c, st2, s2, x2, (Real)op.pad2, y2);
#pragma unroll
            for (int i = 0; i < 4; ++i) y1[i] *= y2[i];
            finish4c<Real, C, false>(op, y1, p, valid, c, nullptr, log_scalers, &acc);
        }
    }
    Real x[4];
    ld4(static_cast<const Real*>(P.op[nops - 1].dest) + ((size_t)p * C + c) * 4, x);
    const double w = catw[c];
    double l = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) l += freqs[i] * (w * (double)x[i]);
#pragma unroll
    for (int o = 1; o < C; o <<= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    double v = 0;
    if (c == 0 && p0 < Pn) {
        double sl = log(l);
        if (cum) {
            sl += acc;
            cum[p0] = acc;
        }
        site[p0] = sl;
        v = sl * patw[p0];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) block[(size_t)blockIdx.x * (kT4 / 32) + threadIdx.x / 32] = v;
}

// The parameter-list walks (variant 7) with each chunk of ops' matrices
// staged in shared memory as k_post4root stages them (variant 14): the
// per-op matrix reads are one-wavefront shared-memory rows instead of
// per-lane global loads of the lane's category.
// One op of the staged walks: op k of the staged chunk, this thread's
// pattern p (stores only when valid).
template <typename Real, int C, bool PRE, bool RANGED>
__device__ __forceinline__ void walk4st_op(const OpDesc& op, const Real* s_m, int k, int c, int p,
                                           bool valid, double* cum, int log_scalers) {
    const bool st2 = op.kind & kX2States;
    Real x2[4];
    int s2 = 0;
    if (st2) s2 = static_cast<const int*>(op.x2)[p];
    else ld4(static_cast<const Real*>(op.x2) + ((size_t)p * C + c) * 4, x2);
    Real y[4], out[4];
    if constexpr (PRE) {
        Real pv[4];
        ld4(static_cast<const Real*>(op.x1) + ((size_t)p * C + c) * 4, pv);
        operand4s<Real, C>(s_m, k, 1, c, st2, s2, x2, (Real)op.pad2, y);
#pragma unroll
        for (int i = 0; i < 4; ++i) y[i] *= pv[i];
#pragma unroll
        for (int j = 0; j < 4; ++j) out[j] = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Real m[4];
            lds4(s_m + mat_row<Real, C>(k, 0, c, i), m);
#pragma unroll
            for (int j = 0; j < 4; ++j) out[j] += m[j] * y[i];
        }
        finish4c<Real, C, RANGED>(op, out, p, valid, c, nullptr, log_scalers);
    } else {
        const bool st1 = op.kind & kX1States;
        Real x1[4];
        int s1 = 0;
        if (st1) s1 = static_cast<const int*>(op.x1)[p];
        else ld4(static_cast<const Real*>(op.x1) + ((size_t)p * C + c) * 4, x1);
        operand4s<Real, C>(s_m, k, 0, c, st1, s1, x1, (Real)op.pad1, out);
        operand4s<Real, C>(s_m, k, 1, c, st2, s2, x2, (Real)op.pad2, y);
#pragma unroll
        for (int i = 0; i < 4; ++i) out[i] *= y[i];
        finish4c<Real, C, RANGED>(op, out, p, valid, c, cum, log_scalers);
    }
}

template <typename Real, int C, bool PRE, bool RANGED>
__global__ void __launch_bounds__(kT4, sizeof(Real) == 4 ? 6 : 1)
k_walk4st(const __grid_constant__ OpParams P, int nops, int Pp, double* cum, int log_scalers) {
    constexpr int K = root_chunk<Real, C>();
    __shared__ __align__(16) Real s_m[K * 2 * C * 16];
    const int c = threadIdx.x % C;
    const int p0 = blockIdx.x * (kT4 / C) + threadIdx.x / C;
    const int p = min(p0, Pp - 1);
    const bool valid = p0 < Pp;
    for (int o0 = 0; o0 < nops; o0 += K) {
        const int n = min(K, nops - o0);
        __syncthreads();
        stage_mats<Real, C, PRE>(s_m, P.op + o0, n);
        __syncthreads();
        for (int k = 0; k < n; ++k)
            walk4st_op<Real, C, PRE, RANGED>(P.op[o0 + k], s_m, k, c, p, valid, cum, log_scalers);
    }
}

// -------------------------------------------------- S = 4, slot walks
// The parameter-list walks with a per-thread cache in shared memory: an op
// whose result a later op of the list reads also writes it to a slot, and the
// reader takes it from there (OpDesc::slots, assigned on the host).  A chain
// of dependent ops then waits on shared memory instead of an L2 round trip
// for the value the same thread stored an op or a few ops before.  Every slot
// row belongs to one thread, so no barriers are needed; the device-memory
// store of every result is kept (the buffers are the API's output).
template <typename Real, int PPT>
__device__ __forceinline__ Real* slot_row(Real* slots, int s, int k) {
    return slots + ((size_t)(s * PPT + k) * kT4 + threadIdx.x) * 4;
}

template <typename Real, int C, int PPT>
__device__ __forceinline__ void post4s_op(const OpDesc& op, Real* slots, int c, int p0,
                                          int pstride, int Pp, double* cum, int log_scalers) {
    const bool st1 = op.kind & kX1States, st2 = op.kind & kX2States;
    const int so = slot_field(op.slots, 0), s1x = slot_field(op.slots, 1),
              s2x = slot_field(op.slots, 2);
    const Real* M1 = static_cast<const Real*>(op.m1) + c * 16;
    const Real* M2 = static_cast<const Real*>(op.m2) + c * 16;
    Real x1[PPT][4], x2[PPT][4];
    int s1[PPT], s2[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int p = min(p0 + k * pstride, Pp - 1);
        if (st1) s1[k] = static_cast<const int*>(op.x1)[p];
        else if (s1x >= 0) ld4(slot_row<Real, PPT>(slots, s1x, k), x1[k]);
        else ld4(static_cast<const Real*>(op.x1) + ((size_t)p * C + c) * 4, x1[k]);
        if (st2) s2[k] = static_cast<const int*>(op.x2)[p];
        else if (s2x >= 0) ld4(slot_row<Real, PPT>(slots, s2x, k), x2[k]);
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
        finish4c<Real, C, false>(op, y1, min(p, Pp - 1), p < Pp, c, cum, log_scalers);
        if (so >= 0) st4(slot_row<Real, PPT>(slots, so, k), y1);
    }
}

template <typename Real, int C, int PPT>
__device__ __forceinline__ void pre4s_op(const OpDesc& op, Real* slots, int c, int p0,
                                         int pstride, int Pp, int log_scalers) {
    const bool st2 = op.kind & kX2States;
    const bool tr = op.kind & kM1Transposed;
    const int so = slot_field(op.slots, 0), s1x = slot_field(op.slots, 1),
              s2x = slot_field(op.slots, 2);
    const Real* M1 = static_cast<const Real*>(op.m1) + c * 16;
    const Real* M2 = static_cast<const Real*>(op.m2) + c * 16;
    Real pv[PPT][4], x2[PPT][4];
    int s2[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int p = min(p0 + k * pstride, Pp - 1);
        if (s1x >= 0) ld4(slot_row<Real, PPT>(slots, s1x, k), pv[k]);
        else ld4(static_cast<const Real*>(op.x1) + ((size_t)p * C + c) * 4, pv[k]);
        if (st2) s2[k] = static_cast<const int*>(op.x2)[p];
        else if (s2x >= 0) ld4(slot_row<Real, PPT>(slots, s2x, k), x2[k]);
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
        finish4c<Real, C, false>(op, out, min(p, Pp - 1), p < Pp, c, nullptr, log_scalers);
        if (so >= 0) st4(slot_row<Real, PPT>(slots, so, k), out);
    }
}

template <typename Real, int C, int PPT, bool PRE>
__global__ void __launch_bounds__(kT4)
k_walk4s(const __grid_constant__ OpParams P, int nops, int Pp, double* cum, int log_scalers) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real* slots = reinterpret_cast<Real*>(smem_raw);
    const int c = threadIdx.x % C;
    const int ppb = kT4 / C;
    const int pstride = gridDim.x * ppb;
    const int p0 = blockIdx.x * ppb + threadIdx.x / C;
    for (int o = 0; o < nops; ++o) {
        if (PRE) pre4s_op<Real, C, PPT>(P.op[o], slots, c, p0, pstride, Pp, log_scalers);
        else post4s_op<Real, C, PPT>(P.op[o], slots, c, p0, pstride, Pp, cum, log_scalers);
    }
}

// ------------------------------------------------ S = 4, grouped walks
// An op list executes in order, but its dependency depth is the tree's
// height, not its length.  The launcher reorders the list by dependency level
// (ops of one level read and write disjoint buffers: no read-after-write,
// write-after-read or write-after-write between them, scale buffers included)
// and cuts each level into groups of at most G ops.  A thread issues the
// operand loads of a whole group before computing any of it, so one memory
// round trip serves G ops: for a 128-taxon tree the pre-order walk's chain of
// 254 dependent steps becomes about 70 with G = 4.  One pattern per thread.
struct GroupParams {
    OpDesc op[kParamOps];
    unsigned char size[kParamOps];      // group size at a group's first op
};

template <typename Real, int C, int G, bool PRE>
__global__ void __launch_bounds__(kT4)
k_walk4g(const __grid_constant__ GroupParams P, int nops, int Pp, double* cum, int log_scalers) {
    const int c = threadIdx.x % C;
    const int p = blockIdx.x * (kT4 / C) + threadIdx.x / C;
    const bool valid = p < Pp;
    const int pc = valid ? p : Pp - 1;
    for (int o = 0; o < nops;) {
        const int g = P.size[o];
        Real a[G][4], b[G][4];
        int s1[G], s2[G];
#pragma unroll
        for (int k = 0; k < G; ++k) {
            if (k < g) {
                const OpDesc& op = P.op[o + k];
                if (!PRE && (op.kind & kX1States)) s1[k] = static_cast<const int*>(op.x1)[pc];
                else ld4(static_cast<const Real*>(op.x1) + ((size_t)pc * C + c) * 4, a[k]);
                if (op.kind & kX2States) s2[k] = static_cast<const int*>(op.x2)[pc];
                else ld4(static_cast<const Real*>(op.x2) + ((size_t)pc * C + c) * 4, b[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < G; ++k) {
            if (k < g) {
                const OpDesc& op = P.op[o + k];
                const Real* M1 = static_cast<const Real*>(op.m1) + c * 16;
                const Real* M2 = static_cast<const Real*>(op.m2) + c * 16;
                const bool st2 = op.kind & kX2States;
                if (!PRE) {
                    Real y1[4], y2[4];
                    operand4c(M1, (op.kind & kX1States) != 0, s1[k], a[k], (Real)op.pad1, y1);
                    operand4c(M2, st2, s2[k], b[k], (Real)op.pad2, y2);
#pragma unroll
                    for (int i = 0; i < 4; ++i) y1[i] *= y2[i];
                    finish4c<Real, C, false>(op, y1, pc, valid, c, cum, log_scalers);
                } else {
                    const bool tr = op.kind & kM1Transposed;
                    Real z[4];
                    operand4c(M2, st2, s2[k], b[k], (Real)op.pad2, z);
#pragma unroll
                    for (int i = 0; i < 4; ++i) z[i] *= a[k][i];
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
                    finish4c<Real, C, false>(op, out, pc, valid, c, nullptr, log_scalers);
                }
            }
        }
        o += g;
    }
}

// ------------------------------------------- S = 4, software-pipelined walk
// Same thread layout as k_post4 / k_pre4, but the loads of op i+1's operands
// are issued before op i is computed, so two ops' loads are in flight per
// thread.  An operand that op i or op i-1 produced is not re-read: every
// thread computes the same (pattern, category) rows in every op, so the value
// is already in its registers (op i's result is forwarded when op i+1 starts,
// op i-1's result is copied at prefetch time).  Operands written earlier than
// that were stored by this same thread before the prefetch load is issued.
//
// Op descriptors are staged in two shared-memory chunks: chunk j+1 is staged
// while chunk j is walked, so the prefetch of the first op of a chunk reads a
// staged descriptor too.
template <typename Real, int PPT>
struct Rows4 {
    Real v[PPT][4];
};

// Load one operand (partials rows or tip states) of PPT patterns.
template <typename Real, int C, int PPT>
__device__ __forceinline__ void load_operand4(const void* x, bool states, const int* pc, int c,
                                              Rows4<Real, PPT>& r, int* st) {
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        if (states) st[k] = static_cast<const int*>(x)[pc[k]];
        else ld4(static_cast<const Real*>(x) + ((size_t)pc[k] * C + c) * 4, r.v[k]);
    }
}

// Where op `nx`'s operand x comes from: 0 = load, 1 = result of the op being
// computed now (`cur_dest`), 2 = result of the op before it (`prev_dest`).  A
// result is forwarded only between ops that write the same pattern range
// (partition): outside its range an op computes values it does not store.
__device__ __forceinline__ int operand_source(const void* x, bool states, const void* cur_dest,
                                              bool cur_same, const void* prev_dest,
                                              bool prev_same) {
    if (states) return 0;
    if (x == cur_dest) return cur_same ? 1 : 0;
    if (x == prev_dest) return prev_same ? 2 : 0;
    return 0;
}

__device__ __forceinline__ const OpDesc& staged_op(const OpDesc* s_ops, int i) {
    return s_ops[((i / kOpChunk) & 1) * kOpChunk + (i % kOpChunk)];
}

// Stage chunk j of the op list into its shared-memory half (j & 1).
__device__ __forceinline__ void stage_chunk(OpDesc* s_ops, const OpDesc* __restrict__ ops,
                                            int nops, int j) {
    const int o0 = j * kOpChunk;
    if (o0 >= nops) return;
    stage_ops(s_ops + (j & 1) * kOpChunk, ops + o0, min(kOpChunk, nops - o0));
}

template <typename Real, int C, int PPT, bool PRE>
__global__ void __launch_bounds__(kT4)
k_walk4_pipe(const OpDesc* __restrict__ ops, int nops, int Pp, double* cum, int log_scalers) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    OpDesc* s_ops = reinterpret_cast<OpDesc*>(smem_raw);      // [2][kOpChunk]
    const int c = threadIdx.x % C;
    const int ppb = kT4 / C;
    const int pstride = gridDim.x * ppb;
    const int p0 = blockIdx.x * ppb + threadIdx.x / C;
    int pc[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) pc[k] = min(p0 + k * pstride, Pp - 1);

    Rows4<Real, PPT> a, b, hist;       // operands of op i; result of op i-1
    int sa[PPT] = {}, sb[PPT] = {};
    int src_a = 0, src_b = 0;          // 1: take the operand from `hist` (op i-1's result)
    const void* prev_dest = nullptr;
    int prev_b = 0, prev_e = 0;        // pattern range of op i-1

    stage_chunk(s_ops, ops, nops, 0);
    __syncthreads();
    {
        const OpDesc& op = staged_op(s_ops, 0);
        load_operand4<Real, C, PPT>(op.x1, !PRE && (op.kind & kX1States), pc, c, a, sa);
        load_operand4<Real, C, PPT>(op.x2, op.kind & kX2States, pc, c, b, sb);
    }
    for (int i = 0; i < nops; ++i) {
        if (i % kOpChunk == 0) {
            // chunk i / kOpChunk is staged; stage the next one into the other half
            // (its previous contents, chunk i / kOpChunk - 1, are no longer read).
            __syncthreads();
            stage_chunk(s_ops, ops, nops, i / kOpChunk + 1);
            __syncthreads();
        }
        const OpDesc& op = staged_op(s_ops, i);
        const bool sta = !PRE && (op.kind & kX1States), stb = op.kind & kX2States;
        // Operands forwarded from op i-1's result.
        if (src_a == 1) a = hist;
        if (src_b == 1) b = hist;
        // Prefetch op i+1's operands.
        Rows4<Real, PPT> na, nb;
        int nsa[PPT] = {}, nsb[PPT] = {};
        int nsrc_a = 0, nsrc_b = 0;
        if (i + 1 < nops) {
            const OpDesc& nx = staged_op(s_ops, i + 1);
            const bool nsta = !PRE && (nx.kind & kX1States), nstb = nx.kind & kX2States;
            const bool cur_same = nx.p_begin == op.p_begin && nx.p_end == op.p_end;
            const bool prev_same = nx.p_begin == prev_b && nx.p_end == prev_e;
            nsrc_a = operand_source(nx.x1, nsta, op.dest, cur_same, prev_dest, prev_same);
            nsrc_b = operand_source(nx.x2, nstb, op.dest, cur_same, prev_dest, prev_same);
            if (nsrc_a == 0) load_operand4<Real, C, PPT>(nx.x1, nsta, pc, c, na, nsa);
            else if (nsrc_a == 2) na = hist;
            if (nsrc_b == 0) load_operand4<Real, C, PPT>(nx.x2, nstb, pc, c, nb, nsb);
            else if (nsrc_b == 2) nb = hist;
        }
        // Compute op i.
        const Real* M1 = static_cast<const Real*>(op.m1) + c * 16;
        const Real* M2 = static_cast<const Real*>(op.m2) + c * 16;
        Rows4<Real, PPT> res;
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            const int p = p0 + k * pstride;
            Real out[4];
            if (!PRE) {
                Real y2[4];
                operand4c(M1, sta, sa[k], a.v[k], (Real)op.pad1, out);
                operand4c(M2, stb, sb[k], b.v[k], (Real)op.pad2, y2);
#pragma unroll
                for (int q = 0; q < 4; ++q) out[q] *= y2[q];
            } else {
                Real z[4];
                operand4c(M2, stb, sb[k], b.v[k], (Real)op.pad2, z);
#pragma unroll
                for (int q = 0; q < 4; ++q) z[q] *= a.v[k][q];
#pragma unroll
                for (int q = 0; q < 4; ++q) out[q] = 0;
                const bool tr = op.kind & kM1Transposed;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    Real m[4];
                    if (tr) {
#pragma unroll
                        for (int j = 0; j < 4; ++j) m[j] = __ldg(M1 + j * 4 + q);
                    } else {
                        ldg4(M1 + q * 4, m);
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) out[j] += m[j] * z[q];
                }
            }
            finish4c<Real, C>(op, out, pc[k], p < Pp, c, PRE ? nullptr : cum, log_scalers);
#pragma unroll
            for (int q = 0; q < 4; ++q) res.v[k][q] = out[q];
        }
        hist = res;
        prev_dest = op.dest;
        prev_b = op.p_begin;
        prev_e = op.p_end;
        a = na;
        b = nb;
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            sa[k] = nsa[k];
            sb[k] = nsb[k];
        }
        src_a = nsrc_a;
        src_b = nsrc_b;
    }
}

// Thread-per-pattern S = 4 kernels for category counts that are not a power
// of two (the lane-group layout above needs C | 32).
template <typename Real, int C>
__device__ __forceinline__ void operand4(const void* x, bool states, const Real* __restrict__ M,
                                         Real pad, int p, Real y[C][4]) {
    if (states) {
        const int s = static_cast<const int*>(x)[p];
#pragma unroll
        for (int c = 0; c < C; ++c) {
#pragma unroll
            for (int i = 0; i < 4; ++i) y[c][i] = (s < 4) ? __ldg(M + c * 16 + i * 4 + s) : pad;
        }
    } else {
        const Real* xp = static_cast<const Real*>(x) + (size_t)p * (C * 4);
        Real xv[C][4];
#pragma unroll
        for (int c = 0; c < C; ++c) ld4(xp + c * 4, xv[c]);
#pragma unroll
        for (int c = 0; c < C; ++c) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                Real m[4];
                ldg4(M + c * 16 + i * 4, m);
                y[c][i] = m[0] * xv[c][0] + m[1] * xv[c][1] + m[2] * xv[c][2] + m[3] * xv[c][3];
            }
        }
    }
}

template <typename Real, int C>
__device__ __forceinline__ void finish4(const OpDesc& op, Real out[C][4], int p,
                                        double* cum, int log_scalers) {
    if (p < op.p_begin || p >= op.p_end) return;
    if (op.cum) cum = op.cum;
    if (op.scale_write) {
        Real m = 0;
#pragma unroll
        for (int c = 0; c < C; ++c)
#pragma unroll
            for (int i = 0; i < 4; ++i) m = out[c][i] > m ? out[c][i] : m;
        if (m == Real(0)) m = Real(1);
        const Real inv = recip(m);
#pragma unroll
        for (int c = 0; c < C; ++c)
#pragma unroll
            for (int i = 0; i < 4; ++i) out[c][i] *= inv;
        store_scale(m, op.scale_write, cum, p, log_scalers);
    } else if (op.scale_read) {
        const Real inv = recip((Real)op.scale_read[p]);
#pragma unroll
        for (int c = 0; c < C; ++c)
#pragma unroll
            for (int i = 0; i < 4; ++i) out[c][i] *= inv;
    }
    Real* d = static_cast<Real*>(op.dest) + (size_t)p * (C * 4);
#pragma unroll
    for (int c = 0; c < C; ++c) st4(d + c * 4, out[c]);
}

template <typename Real, int C>
__global__ void __launch_bounds__(128)
k_post4p(const OpDesc* __restrict__ ops, int nops, int Pp, double* cum, int log_scalers) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Pp) return;
    for (int o = 0; o < nops; ++o) {
        const OpDesc op = ops[o];
        Real y1[C][4], y2[C][4];
        operand4<Real, C>(op.x1, op.kind & kX1States, static_cast<const Real*>(op.m1),
                          (Real)op.pad1, p, y1);
        operand4<Real, C>(op.x2, op.kind & kX2States, static_cast<const Real*>(op.m2),
                          (Real)op.pad2, p, y2);
#pragma unroll
        for (int c = 0; c < C; ++c)
#pragma unroll
            for (int i = 0; i < 4; ++i) y1[c][i] *= y2[c][i];
        finish4<Real, C>(op, y1, p, cum, log_scalers);
    }
}

template <typename Real, int C>
__global__ void __launch_bounds__(128)
k_pre4p(const OpDesc* __restrict__ ops, int nops, int Pp, int log_scalers) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Pp) return;
    for (int o = 0; o < nops; ++o) {
        const OpDesc op = ops[o];
        Real z[C][4];
        operand4<Real, C>(op.x2, op.kind & kX2States, static_cast<const Real*>(op.m2),
                          (Real)op.pad2, p, z);
        const Real* xp = static_cast<const Real*>(op.x1) + (size_t)p * (C * 4);
        const Real* M = static_cast<const Real*>(op.m1);
        const bool tr = op.kind & kM1Transposed;
        Real out[C][4];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            Real pv[4];
            ld4(xp + c * 4, pv);
#pragma unroll
            for (int i = 0; i < 4; ++i) z[c][i] *= pv[i];
#pragma unroll
            for (int j = 0; j < 4; ++j) out[c][j] = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                Real m[4];
                if (tr) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) m[j] = __ldg(M + c * 16 + j * 4 + i);
                } else {
                    ldg4(M + c * 16 + i * 4, m);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) out[c][j] += m[j] * z[c][i];
            }
        }
        finish4<Real, C>(op, out, p, nullptr, log_scalers);
    }
}

// ------------------------------------------------------- batched S = 4 walks
// One launch walks the op lists of several instances with the same category
// count (one pattern per thread, the shape of variant 1).  CTA x belongs to the
// instance whose segment holds x; it walks that instance's list for its own
// patterns, exactly as the single-instance kernel does.
template <typename Seg>
__device__ __forceinline__ int find_walk_seg(const Seg* segs, int nseg, int x) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].first_cta <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The batched walk: CTA x walks the op list (device memory) of the segment
// whose first_cta is the largest one <= x, each chunk's descriptors and
// matrices staged in shared memory together (as k_walk4st).  The segment
// itself stays in shared memory.
template <typename Real, int C, bool PRE>
__global__ void __launch_bounds__(kT4, sizeof(Real) == 4 ? 5 : 1)
k_walk4_batch(const WalkSeg* __restrict__ segs, int nseg) {
    constexpr int K = root_chunk<Real, C>();
    __shared__ OpDesc s_ops[K];
    __shared__ __align__(16) Real s_m[K * 2 * C * 16];
    __shared__ WalkSeg sg;
    if (threadIdx.x == 0) sg = segs[find_walk_seg(segs, nseg, blockIdx.x)];
    __syncthreads();
    const int c = threadIdx.x % C;
    const int p0 = (blockIdx.x - sg.first_cta) * (kT4 / C) + threadIdx.x / C;
    const int Pp = sg.Pp;
    const int p = min(p0, Pp - 1);
    const bool valid = p0 < Pp;
    const int nops = sg.nops;
    for (int o0 = 0; o0 < nops; o0 += K) {
        const int n = min(K, nops - o0);
        __syncthreads();
        stage_ops(s_ops, sg.ops + o0, n);
        stage_mats<Real, C, PRE>(s_m, sg.ops + o0, n);
        __syncthreads();
        for (int k = 0; k < n; ++k)
            walk4st_op<Real, C, PRE, false>(s_ops[k], s_m, k, c, p, valid, PRE ? nullptr : sg.cum,
                                            sg.log_scalers);
    }
}

// k_post4root over many instances: CTA x walks the op list (device memory)
// of the segment whose first_cta is the largest one <= x, each chunk's
// descriptors and matrices staged together as in k_walk4_batch, keeps its
// patterns' log scale factors in registers and forms their site lnL from the
// root row; the member's block partials get one sum per warp.
template <typename Real, int C>
__global__ void __launch_bounds__(kT4, sizeof(Real) == 4 ? 5 : 1)
k_post4root_batch(const PostRootSeg* __restrict__ segs, int nseg) {
    constexpr int K = root_chunk<Real, C>();
    __shared__ OpDesc s_ops[K];
    __shared__ __align__(16) Real s_m[K * 2 * C * 16];
    __shared__ PostRootSeg sg;
    if (threadIdx.x == 0) sg = segs[find_walk_seg(segs, nseg, blockIdx.x)];
    __syncthreads();
    const int c = threadIdx.x % C;
    const int local = blockIdx.x - sg.first_cta;
    const int p0 = local * (kT4 / C) + threadIdx.x / C;
    const int Pp = sg.Pp;
    const int p = min(p0, Pp - 1);
    const bool valid = p0 < Pp;
    const int nops = sg.nops;
    double acc = 0;
    for (int o0 = 0; o0 < nops; o0 += K) {
        const int n = min(K, nops - o0);
        __syncthreads();
        stage_ops(s_ops, sg.ops + o0, n);
        stage_mats<Real, C>(s_m, sg.ops + o0, n);
        __syncthreads();
        for (int k = 0; k < n; ++k) {
            const OpDesc& op = s_ops[k];
            const bool st1 = op.kind & kX1States, st2 = op.kind & kX2States;
            Real x1[4], x2[4];
            int s1 = 0, s2 = 0;
            if (st1) s1 = static_cast<const int*>(op.x1)[p];
            else ld4(static_cast<const Real*>(op.x1) + ((size_t)p * C + c) * 4, x1);
            if (st2) s2 = static_cast<const int*>(op.x2)[p];
            else ld4(static_cast<const Real*>(op.x2) + ((size_t)p * C + c) * 4, x2);
            Real y1[4], y2[4];
            operand4s<Real, C>(s_m, k, 0, c, st1, s1, x1, (Real)op.pad1, y1);
            operand4s<Real, C>(s_m, k, 1, c, st2, s2, x2, (Real)op.pad2, y2);
#pragma unroll
            for (int i = 0; i < 4; ++i) y1[i] *= y2[i];
            finish4c<Real, C, false>(op, y1, p, valid, c, nullptr, sg.log_scalers, &acc);
        }
    }
    Real x[4];
    ld4(static_cast<const Real*>(sg.ops[nops - 1].dest) + ((size_t)p * C + c) * 4, x);
    const double w = sg.catw[c];
    double l = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) l += sg.freqs[i] * (w * (double)x[i]);
#pragma unroll
    for (int o = 1; o < C; o <<= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    double v = 0;
    if (c == 0 && p0 < sg.P) {
        double sl = log(l);
        if (sg.cum) {
            sl += acc;
            sg.cum[p0] = acc;
        }
        sg.site[p0] = sl;
        v = sl * sg.patw[p0];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sg.block[(size_t)local * (kT4 / 32) + threadIdx.x / 32] = v;
}

// Variants of the S = 4 op walks (chosen per shape by the instance's
// autotuner, b200_instance.cpp):
//   0      thread per pattern, all categories in registers (any C <= 8);
//   1,2,3  thread per (pattern, category) with 1, 2 or 4 patterns per thread
//          (C dividing 32);
//   4,5    the software-pipelined walk with 1 or 2 patterns per thread
//          (C dividing 32);
//   6      2 patterns per thread held to <= 42 registers (6 CTAs per SM), so
//          about 110 k patterns of 4 categories fit one resident wave (FP32;
//          FP64 rows need more registers and run as variant 2).
template <typename Real>
constexpr int kMinB6 = sizeof(Real) == 4 ? 6 : 1;
//   7,8    1 or 2 patterns per thread with the op list passed by value as a
//          kernel parameter (one launch per kParamOps ops).
//   9,10   7, 8 with results that later ops read kept in shared-memory slots;
//   11-13  the list reordered by dependency level, groups of 2, 4 or 8
//          independent ops loaded together (one pattern per thread);
//   14     7 with each chunk of ops' matrices staged in shared memory
//          (k_walk4st).
// variant < 0 picks the default: the smallest patterns-per-thread whose grid
// fits in one resident wave, thread per pattern when C does not divide 32.
template <typename K>
long wave_patterns(K kernel, int C, int ppt) {
    int dev = 0, sms = 0, blocks = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, kT4,
                                                  kOpChunk * sizeof(OpDesc));
    return (long)sms * blocks * (kT4 / C) * ppt;
}

template <typename Real, int C>
int default_variant(int Pp, bool pre) {
    if (32 % C != 0) return 0;
    constexpr int CC = (32 % C == 0 ? C : 1);
    static const long p1 = wave_patterns(k_post4<Real, CC, 1, false>, CC, 1);
    static const long p2 = wave_patterns(k_post4<Real, CC, 2, false>, CC, 2);
    static const long q1 = wave_patterns(k_pre4<Real, CC, 1, false>, CC, 1);
    static const long q2 = wave_patterns(k_pre4<Real, CC, 2, false>, CC, 2);
    const long w1 = pre ? q1 : p1, w2 = pre ? q2 : p2;
    return Pp <= w1 ? 1 : Pp <= w2 ? 2 : 3;
}

template <typename Real, int C, int PPT, int MINB = 1>
cudaError_t run_post4_ppt(const OpDesc* ops, int nops, const Dims& d, double* cum, int ls,
                          cudaStream_t s, bool ranged) {
    const int ppb = kT4 / C * PPT;
    const int grid = (d.Pp + ppb - 1) / ppb;
    const size_t sm = kOpChunk * sizeof(OpDesc);
    if (ranged)
        k_post4<Real, C, PPT, true, MINB><<<grid, kT4, sm, s>>>(ops, nops, d.Pp, cum, ls);
    else
        k_post4<Real, C, PPT, false, MINB><<<grid, kT4, sm, s>>>(ops, nops, d.Pp, cum, ls);
    return cudaGetLastError();
}

template <typename Real, int C, int PPT, int MINB = 1>
cudaError_t run_pre4_ppt(const OpDesc* ops, int nops, const Dims& d, int ls, cudaStream_t s,
                         bool ranged) {
    const int ppb = kT4 / C * PPT;
    const int grid = (d.Pp + ppb - 1) / ppb;
    const size_t sm = kOpChunk * sizeof(OpDesc);
    if (ranged) k_pre4<Real, C, PPT, true, MINB><<<grid, kT4, sm, s>>>(ops, nops, d.Pp, ls);
    else k_pre4<Real, C, PPT, false, MINB><<<grid, kT4, sm, s>>>(ops, nops, d.Pp, ls);
    return cudaGetLastError();
}

// Lists longer than kParamOps run as consecutive launches of at most
// kParamOps ops: a launch boundary orders every write of one launch before
// every read of the next, so the cut changes only the launch count.
template <typename Real, int C, int PPT>
cudaError_t run_param4(const OpDesc* h_ops, int nops, const Dims& d, double* cum, int ls,
                       cudaStream_t s, bool ranged, bool pre) {
    if (!h_ops) return cudaErrorInvalidValue;
    static thread_local OpParams prm;    // 28 KB: copied into the launch
    const int ppb = kT4 / C * PPT;
    const int grid = (d.Pp + ppb - 1) / ppb;
    for (int o0 = 0; o0 < nops; o0 += kParamOps) {
        const int n = std::min(kParamOps, nops - o0);
        std::memcpy(prm.op, h_ops + o0, sizeof(OpDesc) * n);
        if (pre) {
            if (ranged) k_pre4c<Real, C, PPT, true><<<grid, kT4, 0, s>>>(prm, n, d.Pp, ls);
            else k_pre4c<Real, C, PPT, false><<<grid, kT4, 0, s>>>(prm, n, d.Pp, ls);
        } else {
            if (ranged) k_post4c<Real, C, PPT, true><<<grid, kT4, 0, s>>>(prm, n, d.Pp, cum, ls);
            else k_post4c<Real, C, PPT, false><<<grid, kT4, 0, s>>>(prm, n, d.Pp, cum, ls);
        }
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Variant 14: the staged walks, one launch per kParamOps ops.
template <typename Real, int C>
cudaError_t run_stage4(const OpDesc* h_ops, int nops, const Dims& d, double* cum, int ls,
                       cudaStream_t s, bool ranged, bool pre) {
    if (!h_ops) return cudaErrorInvalidValue;
    static thread_local OpParams prm;
    const int grid = (d.Pp + kT4 / C - 1) / (kT4 / C);
    for (int o0 = 0; o0 < nops; o0 += kParamOps) {
        const int n = std::min(kParamOps, nops - o0);
        std::memcpy(prm.op, h_ops + o0, sizeof(OpDesc) * n);
        if (pre) {
            if (ranged) k_walk4st<Real, C, true, true><<<grid, kT4, 0, s>>>(prm, n, d.Pp, nullptr, ls);
            else k_walk4st<Real, C, true, false><<<grid, kT4, 0, s>>>(prm, n, d.Pp, nullptr, ls);
        } else {
            if (ranged) k_walk4st<Real, C, false, true><<<grid, kT4, 0, s>>>(prm, n, d.Pp, cum, ls);
            else k_walk4st<Real, C, false, false><<<grid, kT4, 0, s>>>(prm, n, d.Pp, cum, ls);
        }
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Variants 9, 10: the slot walks.  Lists of partition ops carry no slots and
// run as variants 7, 8.
template <typename Real, int C, int PPT>
cudaError_t run_slot4(const OpDesc* h_ops, int nops, const Dims& d, double* cum, int ls,
                      cudaStream_t s, bool ranged, bool pre) {
    if (ranged) return run_param4<Real, C, PPT>(h_ops, nops, d, cum, ls, s, ranged, pre);
    if (!h_ops || nops > kParamOps) return cudaErrorInvalidValue;
    static thread_local OpParams prm;
    std::memcpy(prm.op, h_ops, sizeof(OpDesc) * nops);
    int nslots = 0;
    for (int o = 0; o < nops; ++o)
        for (int f = 0; f < 3; ++f) nslots = std::max(nslots, slot_field(h_ops[o].slots, f) + 1);
    const size_t smem = (size_t)nslots * PPT * kT4 * 4 * sizeof(Real);
    auto kern = pre ? k_walk4s<Real, C, PPT, true> : k_walk4s<Real, C, PPT, false>;
    if (smem > 48 * 1024) {
        const cudaError_t e =
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int ppb = kT4 / C * PPT;
    const int grid = (d.Pp + ppb - 1) / ppb;
    kern<<<grid, kT4, smem, s>>>(prm, nops, d.Pp, pre ? nullptr : cum, ls);
    return cudaGetLastError();
}

// Dependency level of every op of a list (0 = reads nothing an earlier op of
// the list writes): one more than the level of each earlier op it must follow,
// i.e. the last writer of a buffer it reads (partials or scale factors), and
// the last writer and every reader since of a buffer it writes.  Buffers are
// compared by device address.  The shared cumulative scale buffer is an
// accumulation, whose order changes only the rounding of its FP64 sum.
static void op_levels(const OpDesc* ops, int n, std::vector<int>& level) {
    struct Use {
        int written = -1;   // level of the last writer
        int read = -1;      // highest level of a reader
    };
    std::unordered_map<const void*, Use> use;
    use.reserve(4 * n);
    level.assign(n, 0);
    for (int j = 0; j < n; ++j) {
        const OpDesc& op = ops[j];
        const void* rd[3] = {op.x1, op.x2, op.scale_read};
        const void* wr[2] = {op.dest, op.scale_write};
        int L = 0;
        for (const void* q : rd) {
            if (!q) continue;
            auto it = use.find(q);
            if (it != use.end()) L = std::max(L, it->second.written + 1);
        }
        for (const void* q : wr) {
            if (!q) continue;
            auto it = use.find(q);
            if (it != use.end())
                L = std::max(L, std::max(it->second.written, it->second.read) + 1);
        }
        level[j] = L;
        for (const void* q : rd)
            if (q) use[q].read = std::max(use[q].read, L);
        for (const void* q : wr)
            if (q) use[q].written = L;
    }
}

// Variants 11-13: the grouped walks with G = 2, 4, 8.  Lists of partition
// ops run as variant 7.
template <typename Real, int C, int G>
cudaError_t run_group4(const OpDesc* h_ops, int nops, const Dims& d, double* cum, int ls,
                       cudaStream_t s, bool ranged, bool pre) {
    if (ranged) return run_param4<Real, C, 1>(h_ops, nops, d, cum, ls, s, ranged, pre);
    if (!h_ops || nops > kParamOps) return cudaErrorInvalidValue;
    static thread_local GroupParams prm;
    static thread_local std::vector<int> level, order, first;
    op_levels(h_ops, nops, level);
    const int nl = *std::max_element(level.begin(), level.end()) + 1;
    first.assign(nl + 1, 0);                     // counting sort by level (stable)
    for (int j = 0; j < nops; ++j) ++first[level[j] + 1];
    for (int l = 0; l < nl; ++l) first[l + 1] += first[l];
    order.assign(nops, 0);
    for (int j = 0; j < nops; ++j) order[first[level[j]]++] = j;
    int run = 0;
    for (int k = 0; k < nops; ++k) {
        prm.op[k] = h_ops[order[k]];
        prm.size[k] = 0;
        // a group ends at G ops or at a change of level
        if (run == 0 || level[order[k]] != level[order[k - 1]] || run == G) {
            int g = 0;
            while (g < G && k + g < nops && level[order[k + g]] == level[order[k]]) ++g;
            prm.size[k] = (unsigned char)g;
            run = 0;
        }
        ++run;
    }
    const int ppb = kT4 / C;
    const int grid = (d.Pp + ppb - 1) / ppb;
    if (pre) k_walk4g<Real, C, G, true><<<grid, kT4, 0, s>>>(prm, nops, d.Pp, nullptr, ls);
    else k_walk4g<Real, C, G, false><<<grid, kT4, 0, s>>>(prm, nops, d.Pp, cum, ls);
    return cudaGetLastError();
}

template <typename Real, int C, int PPT, bool PRE>
cudaError_t run_pipe4(const OpDesc* ops, int nops, const Dims& d, double* cum, int ls,
                      cudaStream_t s) {
    const int ppb = kT4 / C * PPT;
    const int grid = (d.Pp + ppb - 1) / ppb;
    k_walk4_pipe<Real, C, PPT, PRE><<<grid, kT4, 2 * kOpChunk * sizeof(OpDesc), s>>>(
        ops, nops, d.Pp, cum, ls);
    return cudaGetLastError();
}

template <typename Real, int C>
cudaError_t run_post4(const OpDesc* ops, const OpDesc* h_ops, int nops, const Dims& d,
                      double* cum, int ls, cudaStream_t s, int variant, bool ranged) {
    if (variant < 0) variant = default_variant<Real, C>(d.Pp, false);
    if (variant > 0 && 32 % C == 0) {
        constexpr int CC = (32 % C == 0 ? C : 1);
        switch (variant) {
            case 4: return run_pipe4<Real, CC, 1, false>(ops, nops, d, cum, ls, s);
            case 5: return run_pipe4<Real, CC, 2, false>(ops, nops, d, cum, ls, s);
            case 6: return run_post4_ppt<Real, CC, 2, kMinB6<Real>>(ops, nops, d, cum, ls, s, ranged);
            case 7: return run_param4<Real, CC, 1>(h_ops, nops, d, cum, ls, s, ranged, false);
            case 8: return run_param4<Real, CC, 2>(h_ops, nops, d, cum, ls, s, ranged, false);
            case 9: return run_slot4<Real, CC, 1>(h_ops, nops, d, cum, ls, s, ranged, false);
            case 10: return run_slot4<Real, CC, 2>(h_ops, nops, d, cum, ls, s, ranged, false);
            case 11: return run_group4<Real, CC, 2>(h_ops, nops, d, cum, ls, s, ranged, false);
            case 12: return run_group4<Real, CC, 4>(h_ops, nops, d, cum, ls, s, ranged, false);
            case 13: return run_group4<Real, CC, 8>(h_ops, nops, d, cum, ls, s, ranged, false);
            case 14: return run_stage4<Real, CC>(h_ops, nops, d, cum, ls, s, ranged, false);
            case 1: return run_post4_ppt<Real, CC, 1>(ops, nops, d, cum, ls, s, ranged);
            case 2: return run_post4_ppt<Real, CC, 2>(ops, nops, d, cum, ls, s, ranged);
            default: return run_post4_ppt<Real, CC, 4>(ops, nops, d, cum, ls, s, ranged);
        }
    }
    k_post4p<Real, C><<<(d.Pp + 127) / 128, 128, 0, s>>>(ops, nops, d.Pp, cum, ls);
    return cudaGetLastError();
}

template <typename Real, int C>
cudaError_t run_pre4(const OpDesc* ops, const OpDesc* h_ops, int nops, const Dims& d, int ls,
                     cudaStream_t s, int variant, bool ranged) {
    if (variant < 0) variant = default_variant<Real, C>(d.Pp, true);
    if (variant > 0 && 32 % C == 0) {
        constexpr int CC = (32 % C == 0 ? C : 1);
        switch (variant) {
            case 4: return run_pipe4<Real, CC, 1, true>(ops, nops, d, nullptr, ls, s);
            case 5: return run_pipe4<Real, CC, 2, true>(ops, nops, d, nullptr, ls, s);
            case 6: return run_pre4_ppt<Real, CC, 2, kMinB6<Real>>(ops, nops, d, ls, s, ranged);
            case 7: return run_param4<Real, CC, 1>(h_ops, nops, d, nullptr, ls, s, ranged, true);
            case 8: return run_param4<Real, CC, 2>(h_ops, nops, d, nullptr, ls, s, ranged, true);
            case 9: return run_slot4<Real, CC, 1>(h_ops, nops, d, nullptr, ls, s, ranged, true);
            case 10: return run_slot4<Real, CC, 2>(h_ops, nops, d, nullptr, ls, s, ranged, true);
            case 11: return run_group4<Real, CC, 2>(h_ops, nops, d, nullptr, ls, s, ranged, true);
            case 12: return run_group4<Real, CC, 4>(h_ops, nops, d, nullptr, ls, s, ranged, true);
            case 13: return run_group4<Real, CC, 8>(h_ops, nops, d, nullptr, ls, s, ranged, true);
            case 14: return run_stage4<Real, CC>(h_ops, nops, d, nullptr, ls, s, ranged, true);
            case 1: return run_pre4_ppt<Real, CC, 1>(ops, nops, d, ls, s, ranged);
            case 2: return run_pre4_ppt<Real, CC, 2>(ops, nops, d, ls, s, ranged);
            default: return run_pre4_ppt<Real, CC, 4>(ops, nops, d, ls, s, ranged);
        }
    }
    k_pre4p<Real, C><<<(d.Pp + 127) / 128, 128, 0, s>>>(ops, nops, d.Pp, ls);
    return cudaGetLastError();
}

}  // namespace

int post_root_blocks(const Dims& d) { return (d.Pp + kT4 / d.C - 1) / (kT4 / d.C) * (kT4 / 32); }

template <typename Real>
cudaError_t launch_post4_root(const OpDesc* h_ops, int nops, const Dims& d, double* cum, int ls,
                              const double* catw, const double* freqs, const double* patw,
                              double* site, double* block, double* out, cudaStream_t s) {
    if (d.S != 4 || (d.C != 1 && d.C != 2 && d.C != 4 && d.C != 8) || nops < 1 ||
        nops > kParamOps || !h_ops)
        return cudaErrorInvalidValue;
    static thread_local OpParams prm;
    std::memcpy(prm.op, h_ops, sizeof(OpDesc) * nops);
    const int grid = (d.Pp + kT4 / d.C - 1) / (kT4 / d.C);
#define PR_(CC)                                                                            \
    k_post4root<Real, CC><<<grid, kT4, 0, s>>>(prm, nops, d.Pp, d.P, cum, ls, catw, freqs,  \
                                               patw, site, block)
    switch (d.C) {
        case 1: PR_(1); break;
        case 2: PR_(2); break;
        case 4: PR_(4); break;
        default: PR_(8); break;
    }
#undef PR_
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_final_sum(block, post_root_blocks(d), 1, out, s);
}

template cudaError_t launch_post4_root<float>(const OpDesc*, int, const Dims&, double*, int,
                                              const double*, const double*, const double*,
                                              double*, double*, double*, cudaStream_t);
template cudaError_t launch_post4_root<double>(const OpDesc*, int, const Dims&, double*, int,
                                               const double*, const double*, const double*,
                                               double*, double*, double*, cudaStream_t);

int s4_walk_variants(int C) { return (32 % C == 0) ? 15 : 1; }

template <typename Real>
cudaError_t launch_update_partials(const OpDesc* ops, int nops, const Dims& d, double* cum,
                                   int ls, cudaStream_t s, int variant, bool ranged,
                                   const OpDesc* h_ops) {
    if (nops == 0) return cudaSuccess;
    if (d.S == 4 && d.C <= 8) {
        switch (d.C) {
            case 1: return run_post4<Real, 1>(ops, h_ops, nops, d, cum, ls, s, variant, ranged);
            case 2: return run_post4<Real, 2>(ops, h_ops, nops, d, cum, ls, s, variant, ranged);
            case 3: return run_post4<Real, 3>(ops, h_ops, nops, d, cum, ls, s, variant, ranged);
            case 4: return run_post4<Real, 4>(ops, h_ops, nops, d, cum, ls, s, variant, ranged);
            case 5: return run_post4<Real, 5>(ops, h_ops, nops, d, cum, ls, s, variant, ranged);
            case 6: return run_post4<Real, 6>(ops, h_ops, nops, d, cum, ls, s, variant, ranged);
            case 7: return run_post4<Real, 7>(ops, h_ops, nops, d, cum, ls, s, variant, ranged);
            default: return run_post4<Real, 8>(ops, h_ops, nops, d, cum, ls, s, variant, ranged);
        }
    }
    return cudaErrorInvalidValue;   // other state counts: k_generic.cu
}

template <typename Real>
cudaError_t launch_update_pre_partials(const OpDesc* ops, int nops, const Dims& d, int ls,
                                       cudaStream_t s, int variant, bool ranged,
                                       const OpDesc* h_ops) {
    if (nops == 0) return cudaSuccess;
    if (d.S == 4 && d.C <= 8) {
        switch (d.C) {
            case 1: return run_pre4<Real, 1>(ops, h_ops, nops, d, ls, s, variant, ranged);
            case 2: return run_pre4<Real, 2>(ops, h_ops, nops, d, ls, s, variant, ranged);
            case 3: return run_pre4<Real, 3>(ops, h_ops, nops, d, ls, s, variant, ranged);
            case 4: return run_pre4<Real, 4>(ops, h_ops, nops, d, ls, s, variant, ranged);
            case 5: return run_pre4<Real, 5>(ops, h_ops, nops, d, ls, s, variant, ranged);
            case 6: return run_pre4<Real, 6>(ops, h_ops, nops, d, ls, s, variant, ranged);
            case 7: return run_pre4<Real, 7>(ops, h_ops, nops, d, ls, s, variant, ranged);
            default: return run_pre4<Real, 8>(ops, h_ops, nops, d, ls, s, variant, ranged);
        }
    }
    return cudaErrorInvalidValue;   // other state counts: k_generic.cu
}

int post_root_batch_patterns(int C) { return kT4 / C; }

template <typename Real>
cudaError_t launch_post4_root_batch(const PostRootSeg* d_segs, int nseg, int ncta, int C,
                                    cudaStream_t s) {
    if (nseg == 0 || ncta == 0) return cudaSuccess;
    switch (C) {
        case 1: k_post4root_batch<Real, 1><<<ncta, kT4, 0, s>>>(d_segs, nseg); break;
        case 2: k_post4root_batch<Real, 2><<<ncta, kT4, 0, s>>>(d_segs, nseg); break;
        case 4: k_post4root_batch<Real, 4><<<ncta, kT4, 0, s>>>(d_segs, nseg); break;
        case 8: k_post4root_batch<Real, 8><<<ncta, kT4, 0, s>>>(d_segs, nseg); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template cudaError_t launch_post4_root_batch<float>(const PostRootSeg*, int, int, int,
                                                    cudaStream_t);
template cudaError_t launch_post4_root_batch<double>(const PostRootSeg*, int, int, int,
                                                     cudaStream_t);

// Batched walk: ncta = segs' total CTAs; C in {1, 2, 4, 8}.
template <typename Real>
cudaError_t launch_walk4_batch(const WalkSeg* d_segs, int nseg, int ncta, int C, bool pre,
                               cudaStream_t s) {
    if (nseg == 0 || ncta == 0) return cudaSuccess;
#define WB_(CC)                                                                         \
    (pre ? (k_walk4_batch<Real, CC, true><<<ncta, kT4, 0, s>>>(d_segs, nseg), 0)         \
         : (k_walk4_batch<Real, CC, false><<<ncta, kT4, 0, s>>>(d_segs, nseg), 0))
    switch (C) {
        case 1: WB_(1); break;
        case 2: WB_(2); break;
        case 4: WB_(4); break;
        case 8: WB_(8); break;
        default: return cudaErrorInvalidValue;
    }
#undef WB_
    return cudaGetLastError();
}

template cudaError_t launch_walk4_batch<float>(const WalkSeg*, int, int, int, bool, cudaStream_t);
template cudaError_t launch_walk4_batch<double>(const WalkSeg*, int, int, int, bool, cudaStream_t);

template cudaError_t launch_update_partials<float>(const OpDesc*, int, const Dims&, double*, int,
                                                   cudaStream_t, int, bool, const OpDesc*);
template cudaError_t launch_update_partials<double>(const OpDesc*, int, const Dims&, double*, int,
                                                    cudaStream_t, int, bool, const OpDesc*);
template cudaError_t launch_update_pre_partials<float>(const OpDesc*, int, const Dims&, int,
                                                       cudaStream_t, int, bool, const OpDesc*);
template cudaError_t launch_update_pre_partials<double>(const OpDesc*, int, const Dims&, int,
                                                        cudaStream_t, int, bool, const OpDesc*);

}  // namespace b200
