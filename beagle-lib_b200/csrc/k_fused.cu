// Pre-order partials and the edge derivatives of the same branches in one
// walk (S = 4): beagleB200UpdatePrePartialsWithDerivatives.
//
// The call means updatePrePartials(ops) followed by calculateEdgeDerivatives
// over (post[k], dest of op k) for every op k (CPU/BeagleCPUImpl.hpp:1689-1862
// and :1940-2285).  Run separately, the derivative pass reads back every
// pre-order buffer the walk has just written, and every post-order buffer
// the walk has just read as a sibling.  Here the derivative terms of a branch
// are formed from the registers that hold its new pre-order row, so the
// walk's traffic is the whole cost.
//
// Sibling pairs: the pre-order ops of the two children a, b of one parent
// (consecutive in the list, same parent, each the other's sibling) run as
// one step that loads the parent's row and both children's post-order rows
// once:
//   pre[a] = P_a^T (pre[parent] o P_b post[b]),  pre[b] = P_b^T (pre[parent] o P_a post[a])
// and both branches' derivative terms come from the same registers.
//
// Per branch and pattern (as k_edge_deriv4): n_c = sum_k pre_k (D_c post)_k,
// q_c = sum_k pre_k post_k; d = sum_c w_c n_c / sum_c w_c q_c in the partials'
// precision; the pattern-weighted sums of d and d^2 in FP64.  Each warp
// reduces its patterns' terms and writes one partial sum per branch; the
// final-sum kernel adds them in a fixed order.
//
// Thread per (pattern, category) as in the S = 4 walks; the op list is a
// kernel parameter (constant-bank reads).
#include <algorithm>
#include <cstring>

#include "b200_kernels.h"
#include "b200_vec.cuh"
#include "b200_walk4.cuh"

namespace b200 {

namespace {

constexpr int kFusedOps = 256;
struct FusedParams {
    PreDerivOp op[kFusedOps];
};

template <typename Real, int C>
__device__ __forceinline__ void rescale_store4(const PreDerivOp& op, Real out[4], int p,
                                               bool valid, int c, int log_scalers) {
    if (op.scale_write) {
        Real m = out[0];
#pragma unroll
        for (int i = 1; i < 4; ++i) m = out[i] > m ? out[i] : m;
        m = group_max<C>(m);
        if (m == Real(0)) m = Real(1);
        const Real inv = recip(m);
#pragma unroll
        for (int i = 0; i < 4; ++i) out[i] *= inv;
        if (valid && c == 0) store_scale(m, op.scale_write, nullptr, p, log_scalers);
    }
    if (valid) st4(static_cast<Real*>(op.dest) + ((size_t)p * C + c) * 4, out);
}

// out_j = sum_i M[i][j] z_i (M given transposed when `tr`).
template <typename Real>
__device__ __forceinline__ void apply_node(const Real* M, bool tr, const Real z[4], Real out[4]) {
#pragma unroll
    for (int j = 0; j < 4; ++j) out[j] = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        Real m[4];
        if (tr) {
#pragma unroll
            for (int j = 0; j < 4; ++j) m[j] = __ldg(M + j * 4 + i);
        } else {
            ldg4(M + i * 4, m);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) out[j] += m[j] * z[i];
    }
}

// y = M x for a register-held M (row-major 4 x 4), or column s of M for a tip
// state (pad for the missing state).
template <typename Real>
__device__ __forceinline__ void operand4r(const Real m[16], bool states, int s, const Real x[4],
                                          Real pad, Real y[4]) {
    if (states) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Real v = pad;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (s == j) v = m[i * 4 + j];
            y[i] = v;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            y[i] = m[i * 4] * x[0] + m[i * 4 + 1] * x[1] + m[i * 4 + 2] * x[2] + m[i * 4 + 3] * x[3];
    }
}

// out_j = sum_i m[i][j] z_i for a register-held m.
template <typename Real>
__device__ __forceinline__ void apply_reg(const Real m[16], const Real z[4], Real out[4]) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
        out[j] = m[j] * z[0] + m[4 + j] * z[1] + m[8 + j] * z[2] + m[12 + j] * z[3];
}

// num / den: FP64 division; FP32 through the hardware reciprocal (__fdividef,
// 2 ulp), within the FP32 partials' own error.
__device__ __forceinline__ double quotient(double a, double b) { return a / b; }
__device__ __forceinline__ float quotient(float a, float b) { return __fdividef(a, b); }

// Category-combined derivative value of one pattern for one branch; D is
// this category's derivative matrix (dm, when every op shares one, else the
// op's own, loaded here).
template <typename Real, int C, bool SHARED_D>
__device__ __forceinline__ Real deriv_value(const PreDerivOp& op, const Real dm_shared[16],
                                            const Real pre[4], const Real x[4], int s,
                                            bool states, int c, Real w) {
    Real dm[16];
    if (SHARED_D) {
#pragma unroll
        for (int i = 0; i < 16; ++i) dm[i] = dm_shared[i];
    } else {
        const Real* D = static_cast<const Real*>(op.dmat) + c * 16;
#pragma unroll
        for (int k = 0; k < 4; ++k) ldg4(D + 4 * k, dm + 4 * k);
    }
    Real n = 0, q = 0;
    if (states) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            Real dk = (Real)op.dpad;
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (s == i) dk = dm[k * 4 + i];
            n += pre[k] * dk;
            q += (s >= 4 || k == s) ? pre[k] : Real(0);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const Real y = dm[k * 4] * x[0] + dm[k * 4 + 1] * x[1] + dm[k * 4 + 2] * x[2] +
                           dm[k * 4 + 3] * x[3];
            n += pre[k] * y;
            q += pre[k] * x[k];
        }
    }
    Real num = w * n, den = w * q;
#pragma unroll
    for (int o = 1; o < C; o <<= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
    }
    return quotient(num, den);
}

// Warp sums of the weighted value and its square for branch k (values sit in
// the lanes of category 0, every C-th lane; zero elsewhere); lane 0 writes
// them to this warp's column of the block partials in FP64.  The 32 / C terms
// of one warp are added in the partials' precision: with FP32 partials each
// term already carries FP32 rounding.
template <typename Real, int C>
__device__ __forceinline__ void warp_emit(Real v, Real wp, int k, int nops, int nblk, int wid,
                                          double* block) {
    Real s1 = v * wp, s2 = v * v * wp;
#pragma unroll
    for (int o = C; o < 32; o <<= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        block[(size_t)k * nblk + wid] = (double)s1;
        block[(size_t)(nops + k) * nblk + wid] = (double)s2;
    }
}

// As warp_emit, for terms already weighted: (sum w d, sum w d^2).
template <typename Real, int C>
__device__ __forceinline__ void warp_emit2(Real s1, Real s2, int k, int nops, int nblk, int wid,
                                           double* block) {
#pragma unroll
    for (int o = C; o < 32; o <<= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        block[(size_t)k * nblk + wid] = (double)s1;
        block[(size_t)(nops + k) * nblk + wid] = (double)s2;
    }
}

template <typename Real>
__device__ __forceinline__ void load_row(const void* x, bool states, int pc, int C, int c,
                                         Real v[4], int& s) {
    if (states) s = static_cast<const int*>(x)[pc];
    else ld4(static_cast<const Real*>(x) + ((size_t)pc * C + c) * 4, v);
}

// MATS: every sibling pair's two ops use the same two matrices (kPairMats),
// held in registers.  Resident CTAs per SM: FP32 4 (64 registers a thread),
// 3 with matrices or the shared derivative matrix in registers; FP64 2.
template <typename Real, int C, bool SHARED_D, bool MATS>
__global__ void __launch_bounds__(kT4, sizeof(Real) == 4 ? (SHARED_D || MATS ? 3 : 4) : 2)
k_pre_deriv4(const __grid_constant__ FusedParams F, int nops, int P, int Pp,
             const double* __restrict__ catw, const double* __restrict__ patw, int log_scalers,
             double* block) {
    const int c = threadIdx.x % C;
    Real dm[16];
    if (SHARED_D) {
        const Real* D = static_cast<const Real*>(F.op[0].dmat) + c * 16;
#pragma unroll
        for (int k = 0; k < 4; ++k) ldg4(D + 4 * k, dm + 4 * k);
    }
    const int p = blockIdx.x * (kT4 / C) + threadIdx.x / C;
    const bool valid = p < Pp;
    const int pc = valid ? p : Pp - 1;
    const Real w = (Real)catw[c];
    const bool counted = c == 0 && p < P;
    const Real wp = counted ? (Real)patw[p] : Real(0);
    const int nblk = gridDim.x * (kT4 / 32);
    const int wid = blockIdx.x * (kT4 / 32) + threadIdx.x / 32;
    for (int o = 0; o < nops;) {
        const PreDerivOp& A = F.op[o];
        const bool tra = A.kind & kM1Transposed;
        Real pv[4];
        ld4(static_cast<const Real*>(A.parent) + ((size_t)pc * C + c) * 4, pv);
        if (A.kind & kPairFirst) {
            const PreDerivOp& B = F.op[o + 1];
            const bool sta = A.kind & kPostStates, stb = A.kind & kX2States;
            Real xa[4], xb[4];
            int sa = 0, sb = 0;
            load_row(A.post, sta, pc, C, c, xa, sa);     // post[a] (= B's sibling)
            load_row(A.sib, stb, pc, C, c, xb, sb);      // post[b] (= A's sibling)
            Real ya[4], yb[4], za[4], zb[4], pa[4], pb[4];
            if (MATS) {
                // P_a and P_b serve both ops: loaded once, kept in registers
                Real ma[16], mb[16];
                const Real* Ma = static_cast<const Real*>(A.mnode) + c * 16;
                const Real* Mb = static_cast<const Real*>(A.msib) + c * 16;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    ldg4(Ma + 4 * k, ma + 4 * k);
                    ldg4(Mb + 4 * k, mb + 4 * k);
                }
                operand4r(mb, stb, sb, xb, (Real)A.pad_sib, yb);
                operand4r(ma, sta, sa, xa, (Real)B.pad_sib, ya);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    za[i] = pv[i] * yb[i];
                    zb[i] = pv[i] * ya[i];
                }
                apply_reg(ma, za, pa);
                apply_reg(mb, zb, pb);
            } else {
                operand4c(static_cast<const Real*>(A.msib) + c * 16, stb, sb, xb,
                          (Real)A.pad_sib, yb);
                operand4c(static_cast<const Real*>(B.msib) + c * 16, sta, sa, xa,
                          (Real)B.pad_sib, ya);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    za[i] = pv[i] * yb[i];
                    zb[i] = pv[i] * ya[i];
                }
                apply_node(static_cast<const Real*>(A.mnode) + c * 16, tra, za, pa);
                apply_node(static_cast<const Real*>(B.mnode) + c * 16,
                           (B.kind & kM1Transposed) != 0, zb, pb);
            }
            rescale_store4<Real, C>(A, pa, pc, valid, c, log_scalers);
            rescale_store4<Real, C>(B, pb, pc, valid, c, log_scalers);
            Real da, db;
            if (!SHARED_D && (A.kind & kPairD)) {
                // one derivative matrix for both branches: loaded once
                Real dp[16];
                const Real* D = static_cast<const Real*>(A.dmat) + c * 16;
#pragma unroll
                for (int k = 0; k < 4; ++k) ldg4(D + 4 * k, dp + 4 * k);
                da = deriv_value<Real, C, true>(A, dp, pa, xa, sa, sta, c, w);
                db = deriv_value<Real, C, true>(B, dp, pb, xb, sb, stb, c, w);
            } else {
                da = deriv_value<Real, C, SHARED_D>(A, dm, pa, xa, sa, sta, c, w);
                db = deriv_value<Real, C, SHARED_D>(B, dm, pb, xb, sb, stb, c, w);
            }
            warp_emit<Real, C>(counted ? da : Real(0), wp, o, nops, nblk, wid, block);
            warp_emit<Real, C>(counted ? db : Real(0), wp, o + 1, nops, nblk, wid, block);
            o += 2;
        } else {
            const bool sts = A.kind & kX2States, stp = A.kind & kPostStates;
            Real xs[4], xp[4];
            int ss = 0, sp = 0;
            load_row(A.sib, sts, pc, C, c, xs, ss);
            load_row(A.post, stp, pc, C, c, xp, sp);
            Real y[4], z[4], pa[4];
            operand4c(static_cast<const Real*>(A.msib) + c * 16, sts, ss, xs, (Real)A.pad_sib, y);
#pragma unroll
            for (int i = 0; i < 4; ++i) z[i] = pv[i] * y[i];
            apply_node(static_cast<const Real*>(A.mnode) + c * 16, tra, z, pa);
            rescale_store4<Real, C>(A, pa, pc, valid, c, log_scalers);
            const Real da = deriv_value<Real, C, SHARED_D>(A, dm, pa, xp, sp, stp, c, w);
            warp_emit<Real, C>(counted ? da : Real(0), wp, o, nops, nblk, wid, block);
            o += 1;
        }
    }
}

// Lists made only of sibling pairs that share their matrices and derivative
// matrix (kPairFirst | kPairMats | kPairD on every even op), FP32: PPT
// patterns per thread (p, p + grid stride, ...), so each pair step's matrix
// loads, descriptor reads and warp reductions serve PPT patterns.
template <int C, int PPT>
__global__ void __launch_bounds__(kT4, 2)
k_pre_deriv4_pairs(const __grid_constant__ FusedParams F, int nops, int P, int Pp,
                   const double* __restrict__ catw, const double* __restrict__ patw,
                   int log_scalers, double* block) {
    using Real = float;
    const int c = threadIdx.x % C;
    const int pstride = gridDim.x * (kT4 / C);
    const int p0 = blockIdx.x * (kT4 / C) + threadIdx.x / C;
    int pc[PPT];
    bool valid[PPT];
    Real wp[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        const int p = p0 + k * pstride;
        valid[k] = p < Pp;
        pc[k] = valid[k] ? p : Pp - 1;
        wp[k] = (c == 0 && p < P) ? (Real)patw[p] : Real(0);
    }
    const Real w = (Real)catw[c];
    const int nblk = gridDim.x * (kT4 / 32);
    const int wid = blockIdx.x * (kT4 / 32) + threadIdx.x / 32;
    for (int o = 0; o < nops; o += 2) {
        const PreDerivOp& A = F.op[o];
        const PreDerivOp& B = F.op[o + 1];
        const bool sta = A.kind & kPostStates, stb = A.kind & kX2States;
        Real ma[16], mb[16];
        const Real* Ma = static_cast<const Real*>(A.mnode) + c * 16;
        const Real* Mb = static_cast<const Real*>(A.msib) + c * 16;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            ldg4(Ma + 4 * k, ma + 4 * k);
            ldg4(Mb + 4 * k, mb + 4 * k);
        }
        Real pa[PPT][4], pb[PPT][4], xa[PPT][4], xb[PPT][4];
        int sa[PPT], sb[PPT];
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            Real pv[4], ya[4], yb[4], za[4], zb[4];
            ld4(static_cast<const Real*>(A.parent) + ((size_t)pc[k] * C + c) * 4, pv);
            sa[k] = sb[k] = 0;
            load_row(A.post, sta, pc[k], C, c, xa[k], sa[k]);
            load_row(A.sib, stb, pc[k], C, c, xb[k], sb[k]);
            operand4r(mb, stb, sb[k], xb[k], (Real)A.pad_sib, yb);
            operand4r(ma, sta, sa[k], xa[k], (Real)B.pad_sib, ya);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                za[i] = pv[i] * yb[i];
                zb[i] = pv[i] * ya[i];
            }
            apply_reg(ma, za, pa[k]);
            apply_reg(mb, zb, pb[k]);
            rescale_store4<Real, C>(A, pa[k], pc[k], valid[k], c, log_scalers);
            rescale_store4<Real, C>(B, pb[k], pc[k], valid[k], c, log_scalers);
        }
        Real dp[16];
        const Real* D = static_cast<const Real*>(A.dmat) + c * 16;
#pragma unroll
        for (int k = 0; k < 4; ++k) ldg4(D + 4 * k, dp + 4 * k);
        Real a1 = 0, a2 = 0, b1 = 0, b2 = 0;
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            const Real da = deriv_value<Real, C, true>(A, dp, pa[k], xa[k], sa[k], sta, c, w);
            const Real db = deriv_value<Real, C, true>(B, dp, pb[k], xb[k], sb[k], stb, c, w);
            const Real ea = wp[k] != Real(0) ? da : Real(0);
            const Real eb = wp[k] != Real(0) ? db : Real(0);
            a1 += ea * wp[k];
            a2 += ea * ea * wp[k];
            b1 += eb * wp[k];
            b2 += eb * eb * wp[k];
        }
        warp_emit2<Real, C>(a1, a2, o, nops, nblk, wid, block);
        warp_emit2<Real, C>(b1, b2, o + 1, nops, nblk, wid, block);
    }
}

// ------------------------------------------------- staged-matrix fused walk
// The fused walk with each op's three matrices in shared memory instead of
// registers or per-lane global loads.  A chunk of ops' matrices is copied
// into shared memory by the whole CTA, each in the orientation its op reads
// it, as rows of 4 values:
//   node   rows of P (the op's matrix given transposed is turned back), for
//          out_j = sum_i P[i][j] z_i;
//   sib    rows of P_sib for a partials sibling (y = P_sib x), its
//          transpose for a tip sibling (column s = one row);
//   deriv  rows of D for a partials post-order row, its transpose for a tip.
// Within a category's 4 rows the order is rotated by c / 2, so the lanes of
// one pattern group (one category each) reading the same row index hit
// distinct banks.  Chunks never split a sibling pair.
template <typename Real, int C>
constexpr int fused_chunk() {
    return 12288 / (3 * C * 16 * (int)sizeof(Real)) < 32 ? 12288 / (3 * C * 16 * (int)sizeof(Real))
                                                         : 32;
}

template <int C>
__device__ __forceinline__ int mat3_row(int k, int w, int c, int i) {
    return (((k * 3 + w) * C + c) * 4 + ((i + (c >> 1)) & 3)) * 4;
}

template <typename Real>
__device__ __forceinline__ void lds4(const Real* r, Real m[4]) {
    if constexpr (sizeof(Real) == 4) {
        const float4 q = *reinterpret_cast<const float4*>(r);
        m[0] = q.x; m[1] = q.y; m[2] = q.z; m[3] = q.w;
    } else {
        const double2 a = reinterpret_cast<const double2*>(r)[0];
        const double2 b = reinterpret_cast<const double2*>(r)[1];
        m[0] = a.x; m[1] = a.y; m[2] = b.x; m[3] = b.y;
    }
}

template <typename Real, int C>
__device__ __forceinline__ void stage_mats3(Real* sm, const PreDerivOp* ops, int n) {
    for (int u = threadIdx.x; u < n * 3 * C * 4; u += kT4) {
        const int i = u & 3, c = (u >> 2) % C, w = (u / (4 * C)) % 3, k = u / (12 * C);
        const PreDerivOp& op = ops[k];
        const void* src = w == 0 ? op.mnode : w == 1 ? op.msib : op.dmat;
        const bool tr = w == 0 ? (op.kind & kM1Transposed) != 0
                      : w == 1 ? (op.kind & kX2States) != 0
                               : (op.kind & kPostStates) != 0;
        const Real* M = static_cast<const Real*>(src) + c * 16;
        Real v[4];
        if (tr) {
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = __ldg(M + j * 4 + i);
        } else {
            ldg4(M + i * 4, v);
        }
        Real* d = sm + mat3_row<C>(k, w, c, i);
#pragma unroll
        for (int j = 0; j < 4; ++j) d[j] = v[j];
    }
}

// y = P_sib x, or column s of P_sib for a tip (pad for the missing state).
template <typename Real, int C>
__device__ __forceinline__ void sib_operand(const Real* sm, int k, int c, bool states, int s,
                                            const Real x[4], Real pad, Real y[4]) {
    if (states) {
        lds4(sm + mat3_row<C>(k, 1, c, s & 3), y);
#pragma unroll
        for (int i = 0; i < 4; ++i) y[i] = s < 4 ? y[i] : pad;
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Real m[4];
            lds4(sm + mat3_row<C>(k, 1, c, i), m);
            y[i] = m[0] * x[0] + m[1] * x[1] + m[2] * x[2] + m[3] * x[3];
        }
    }
}

// out_j = sum_i P[i][j] z_i.
template <typename Real, int C>
__device__ __forceinline__ void node_apply(const Real* sm, int k, int c, const Real z[4],
                                           Real out[4]) {
#pragma unroll
    for (int j = 0; j < 4; ++j) out[j] = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        Real m[4];
        lds4(sm + mat3_row<C>(k, 0, c, i), m);
#pragma unroll
        for (int j = 0; j < 4; ++j) out[j] += m[j] * z[i];
    }
}

// deriv_value with D's rows (or its transpose's, for a tip) from the chunk.
template <typename Real, int C>
__device__ __forceinline__ Real deriv_staged(const Real* sm, int k, Real dpad, const Real pre[4],
                                             const Real x[4], int s, bool states, int c, Real w) {
    Real n = 0, q = 0;
    if (states) {
        Real d[4];
        lds4(sm + mat3_row<C>(k, 2, c, s & 3), d);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            n += pre[j] * (s < 4 ? d[j] : dpad);
            q += (s >= 4 || j == s) ? pre[j] : Real(0);
        }
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            Real m[4];
            lds4(sm + mat3_row<C>(k, 2, c, j), m);
            const Real y = m[0] * x[0] + m[1] * x[1] + m[2] * x[2] + m[3] * x[3];
            n += pre[j] * y;
            q += pre[j] * x[j];
        }
    }
    Real num = w * n, den = w * q;
#pragma unroll
    for (int o = 1; o < C; o <<= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
    }
    return quotient(num, den);
}

// warp_emit for the two branches of a sibling pair at once: the four sums
// (w d and w d^2 of branches k and k + 1) are reduced over the warp's
// patterns by recursive halving -- at the first two levels each lane passes
// on half of what it holds -- so 3 + log2(32 / C) - 2 shuffles replace
// 4 log2(32 / C); lanes 0, C, 2C, 3C then hold one sum each and store it.
template <typename Real, int C>
__device__ __forceinline__ void warp_emit_pair(Real va, Real vb, Real wp, int k, int nops,
                                               int nblk, int wid, double* block) {
    const int lane = threadIdx.x & 31;
    const bool h1 = lane & C, h2 = lane & (2 * C);
    const Real a1 = va * wp, a2 = va * va * wp, b1 = vb * wp, b2 = vb * vb * wp;
    // level 1: lanes with h1 keep branch k + 1's sums, the others branch k's
    Real u0 = h1 ? b1 : a1, u1 = h1 ? b2 : a2;
    u0 += __shfl_xor_sync(0xffffffffu, h1 ? a1 : b1, C);
    u1 += __shfl_xor_sync(0xffffffffu, h1 ? a2 : b2, C);
    // level 2: lanes with h2 keep the square sum, the others the plain sum
    Real v = h2 ? u1 : u0;
    v += __shfl_xor_sync(0xffffffffu, h2 ? u0 : u1, 2 * C);
#pragma unroll
    for (int o = 4 * C; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane < 4 * C && lane % C == 0)
        block[(size_t)((h2 ? nops : 0) + k + (h1 ? 1 : 0)) * nblk + wid] = (double)v;
}

// L2 prefetch (a hint) of this thread's row of a partials operand, or of its
// pattern's entry of a tip-state array.
template <typename Real, int C>
__device__ __forceinline__ void prefetch_row(const void* x, bool states, int pc, int c) {
    const void* a = states ? static_cast<const void*>(static_cast<const int*>(x) + pc)
                           : static_cast<const void*>(static_cast<const Real*>(x) +
                                                      ((size_t)pc * C + c) * 4);
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
}

template <typename Real, int C>
__global__ void __launch_bounds__(kT4, sizeof(Real) == 4 ? 4 : 2)
k_pre_deriv4s(const __grid_constant__ FusedParams F, int nops, int P, int Pp,
              const double* __restrict__ catw, const double* __restrict__ patw, int log_scalers,
              double* block) {
    constexpr int K = fused_chunk<Real, C>();
    __shared__ __align__(16) Real s_m[K * 3 * C * 16];
    const int c = threadIdx.x % C;
    const int p = blockIdx.x * (kT4 / C) + threadIdx.x / C;
    const bool valid = p < Pp;
    const int pc = valid ? p : Pp - 1;
    const Real w = (Real)catw[c];
    const bool counted = c == 0 && p < P;
    const Real wp = counted ? (Real)patw[p] : Real(0);
    const int nblk = gridDim.x * (kT4 / 32);
    const int wid = blockIdx.x * (kT4 / 32) + threadIdx.x / 32;
    for (int o0 = 0; o0 < nops;) {
        int n = min(K, nops - o0);
        if (o0 + n < nops && (F.op[o0 + n - 1].kind & kPairFirst)) --n;
        __syncthreads();
        stage_mats3<Real, C>(s_m, F.op + o0, n);
        __syncthreads();
        for (int k = 0; k < n;) {
            const PreDerivOp& A = F.op[o0 + k];
            Real pv[4];
            ld4(static_cast<const Real*>(A.parent) + ((size_t)pc * C + c) * 4, pv);
            {
                // the next step's post-order operands (written by the post-order
                // walk long before, so read from DRAM) into L2 a step ahead
                const int kn = o0 + k + ((A.kind & kPairFirst) ? 2 : 1);
                if (kn < nops) {
                    const PreDerivOp& An = F.op[kn];
                    prefetch_row<Real, C>(An.post, (An.kind & kPostStates) != 0, pc, c);
                    prefetch_row<Real, C>(An.sib, (An.kind & kX2States) != 0, pc, c);
                }
            }
            if (A.kind & kPairFirst) {
                const PreDerivOp& B = F.op[o0 + k + 1];
                const bool sta = A.kind & kPostStates, stb = A.kind & kX2States;
                Real xa[4], xb[4];
                int sa = 0, sb = 0;
                load_row(A.post, sta, pc, C, c, xa, sa);     // post[a] (= B's sibling)
                load_row(A.sib, stb, pc, C, c, xb, sb);      // post[b] (= A's sibling)
                Real y[4], z[4], pa[4], pb[4];
                sib_operand<Real, C>(s_m, k, c, stb, sb, xb, (Real)A.pad_sib, y);
#pragma unroll
                for (int i = 0; i < 4; ++i) z[i] = pv[i] * y[i];
                node_apply<Real, C>(s_m, k, c, z, pa);
                sib_operand<Real, C>(s_m, k + 1, c, sta, sa, xa, (Real)B.pad_sib, y);
#pragma unroll
                for (int i = 0; i < 4; ++i) z[i] = pv[i] * y[i];
                node_apply<Real, C>(s_m, k + 1, c, z, pb);
                rescale_store4<Real, C>(A, pa, pc, valid, c, log_scalers);
                rescale_store4<Real, C>(B, pb, pc, valid, c, log_scalers);
                const Real da =
                    deriv_staged<Real, C>(s_m, k, (Real)A.dpad, pa, xa, sa, sta, c, w);
                const Real db =
                    deriv_staged<Real, C>(s_m, k + 1, (Real)B.dpad, pb, xb, sb, stb, c, w);
                warp_emit_pair<Real, C>(counted ? da : Real(0), counted ? db : Real(0), wp,
                                        o0 + k, nops, nblk, wid, block);
                k += 2;
            } else {
                const bool sts = A.kind & kX2States, stp = A.kind & kPostStates;
                Real xs[4], xp[4];
                int ss = 0, sp = 0;
                load_row(A.sib, sts, pc, C, c, xs, ss);
                load_row(A.post, stp, pc, C, c, xp, sp);
                Real y[4], z[4], pa[4];
                sib_operand<Real, C>(s_m, k, c, sts, ss, xs, (Real)A.pad_sib, y);
#pragma unroll
                for (int i = 0; i < 4; ++i) z[i] = pv[i] * y[i];
                node_apply<Real, C>(s_m, k, c, z, pa);
                rescale_store4<Real, C>(A, pa, pc, valid, c, log_scalers);
                const Real da =
                    deriv_staged<Real, C>(s_m, k, (Real)A.dpad, pa, xp, sp, stp, c, w);
                warp_emit<Real, C>(counted ? da : Real(0), wp, o0 + k, nops, nblk, wid, block);
                k += 1;
            }
        }
        o0 += n;
    }
}

// ------------------------------------------------------ batched fused walk
// The staged fused walk over several instances with one category count: CTA
// x belongs to the segment whose first_cta is the largest one <= x, and walks
// that instance's op list (device memory): each chunk's descriptors and
// matrices are staged in shared memory together, chunks never splitting a
// sibling pair.  Per op the arithmetic of k_pre_deriv4s.  The segment itself
// stays in shared memory; its fields are read where they are used.
template <typename Real, int C>
__global__ void __launch_bounds__(kT4, sizeof(Real) == 4 ? 4 : 2)
k_pre_deriv4_batch(const PreDerivSeg* __restrict__ segs, int nseg) {
    constexpr int K = fused_chunk<Real, C>();
    __shared__ PreDerivOp s_ops[K];
    __shared__ __align__(16) Real s_m[K * 3 * C * 16];
    __shared__ PreDerivSeg sg;
    if (threadIdx.x == 0) {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (segs[mid].first_cta <= (int)blockIdx.x) lo = mid;
            else hi = mid - 1;
        }
        sg = segs[lo];
    }
    __syncthreads();
    const int c = threadIdx.x % C;
    const int local = blockIdx.x - sg.first_cta;
    const int p = local * (kT4 / C) + threadIdx.x / C;
    const int Pp = sg.Pp;
    const bool valid = p < Pp;
    const int pc = valid ? p : Pp - 1;
    const Real w = (Real)sg.catw[c];
    const bool counted = c == 0 && p < sg.P;
    const Real wp = counted ? (Real)sg.patw[p] : Real(0);
    const int wid = local * (kT4 / 32) + threadIdx.x / 32;
    const int nops = sg.nops;
    for (int o0 = 0; o0 < nops;) {
        const PreDerivOp* fops = sg.fops + o0;
        int n = min(K, nops - o0);
        if (o0 + n < nops && (fops[n - 1].kind & kPairFirst)) --n;
        __syncthreads();
        {
            const int* src = reinterpret_cast<const int*>(fops);
            int* dst = reinterpret_cast<int*>(s_ops);
            const int words = n * (int)(sizeof(PreDerivOp) / sizeof(int));
            for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
        }
        stage_mats3<Real, C>(s_m, fops, n);
        __syncthreads();
        for (int k = 0; k < n;) {
            const PreDerivOp& A = s_ops[k];
            Real pv[4];
            ld4(static_cast<const Real*>(A.parent) + ((size_t)pc * C + c) * 4, pv);
            if (A.kind & kPairFirst) {
                const PreDerivOp& B = s_ops[k + 1];
                const bool sta = A.kind & kPostStates, stb = A.kind & kX2States;
                Real xa[4], xb[4];
                int sa = 0, sb = 0;
                load_row(A.post, sta, pc, C, c, xa, sa);
                load_row(A.sib, stb, pc, C, c, xb, sb);
                Real y[4], z[4], pa[4], pb[4];
                sib_operand<Real, C>(s_m, k, c, stb, sb, xb, (Real)A.pad_sib, y);
#pragma unroll
                for (int i = 0; i < 4; ++i) z[i] = pv[i] * y[i];
                node_apply<Real, C>(s_m, k, c, z, pa);
                sib_operand<Real, C>(s_m, k + 1, c, sta, sa, xa, (Real)B.pad_sib, y);
#pragma unroll
                for (int i = 0; i < 4; ++i) z[i] = pv[i] * y[i];
                node_apply<Real, C>(s_m, k + 1, c, z, pb);
                rescale_store4<Real, C>(A, pa, pc, valid, c, sg.log_scalers);
                rescale_store4<Real, C>(B, pb, pc, valid, c, sg.log_scalers);
                const Real da =
                    deriv_staged<Real, C>(s_m, k, (Real)A.dpad, pa, xa, sa, sta, c, w);
                const Real db =
                    deriv_staged<Real, C>(s_m, k + 1, (Real)B.dpad, pb, xb, sb, stb, c, w);
                warp_emit_pair<Real, C>(counted ? da : Real(0), counted ? db : Real(0), wp,
                                        o0 + k, nops, sg.nblk, wid, sg.block);
                k += 2;
            } else {
                const bool sts = A.kind & kX2States, stp = A.kind & kPostStates;
                Real xs[4], xp[4];
                int ss = 0, sp = 0;
                load_row(A.sib, sts, pc, C, c, xs, ss);
                load_row(A.post, stp, pc, C, c, xp, sp);
                Real y[4], z[4], pa[4];
                sib_operand<Real, C>(s_m, k, c, sts, ss, xs, (Real)A.pad_sib, y);
#pragma unroll
                for (int i = 0; i < 4; ++i) z[i] = pv[i] * y[i];
                node_apply<Real, C>(s_m, k, c, z, pa);
                rescale_store4<Real, C>(A, pa, pc, valid, c, sg.log_scalers);
                const Real da =
                    deriv_staged<Real, C>(s_m, k, (Real)A.dpad, pa, xp, sp, stp, c, w);
                warp_emit<Real, C>(counted ? da : Real(0), wp, o0 + k, nops, sg.nblk, wid,
                                   sg.block);
                k += 1;
            }
        }
        o0 += n;
    }
}

}  // namespace

int pre_deriv4_batch_patterns(int C) { return kT4 / C; }

template <typename Real>
cudaError_t launch_pre_deriv4_batch(const PreDerivSeg* d_segs, int nseg, int ncta, int C,
                                    cudaStream_t s) {
    if (nseg == 0 || ncta == 0) return cudaSuccess;
    switch (C) {
        case 1: k_pre_deriv4_batch<Real, 1><<<ncta, kT4, 0, s>>>(d_segs, nseg); break;
        case 2: k_pre_deriv4_batch<Real, 2><<<ncta, kT4, 0, s>>>(d_segs, nseg); break;
        case 4: k_pre_deriv4_batch<Real, 4><<<ncta, kT4, 0, s>>>(d_segs, nseg); break;
        case 8: k_pre_deriv4_batch<Real, 8><<<ncta, kT4, 0, s>>>(d_segs, nseg); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template cudaError_t launch_pre_deriv4_batch<float>(const PreDerivSeg*, int, int, int,
                                                    cudaStream_t);
template cudaError_t launch_pre_deriv4_batch<double>(const PreDerivSeg*, int, int, int,
                                                     cudaStream_t);

int fused_blocks(const Dims& d) { return (d.Pp + kT4 / d.C - 1) / (kT4 / d.C) * (kT4 / 32); }

bool fused_supported(const Dims& d, int /*nops*/) {
    return d.S == 4 && d.Sg == 4 && (d.C == 1 || d.C == 2 || d.C == 4 || d.C == 8);
}

namespace {

// One launch of the fused walk over at most kFusedOps ops; the sums of op k
// go to d_sums[k] and d_sums[nsum + k] (nsum: the whole list's length).
template <typename Real>
cudaError_t pre_deriv4_chunk(const PreDerivOp* h_ops, int nops, const Dims& d,
                             const double* catw, const double* patw, int ls, double* d_block,
                             double* d_sums, int nsum, cudaStream_t s, int variant) {
    static thread_local FusedParams prm;   // copied into the launch
    std::memcpy(prm.op, h_ops, sizeof(PreDerivOp) * nops);
    auto final_sums = [&](int nblk) {
        if (nsum == nops) return launch_deriv_final(d_block, nblk, nops, d_sums, s);
        return launch_deriv_final_at(d_block, nblk, nops, d_sums, d_sums + nsum, s);
    };
    if (variant == 2) {
        // pairs-only lists, FP32, 2 patterns per thread
        constexpr int kAll = kPairFirst | kPairMats | kPairD;
        if (sizeof(Real) != 4 || nops % 2) return cudaErrorInvalidValue;
        for (int k = 0; k < nops; k += 2)
            if ((h_ops[k].kind & kAll) != kAll) return cudaErrorInvalidValue;
        const int grid2 = (d.Pp + 2 * (kT4 / d.C) - 1) / (2 * (kT4 / d.C));
        switch (d.C) {
            case 1: k_pre_deriv4_pairs<1, 2><<<grid2, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw, patw, ls, d_block); break;
            case 2: k_pre_deriv4_pairs<2, 2><<<grid2, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw, patw, ls, d_block); break;
            case 4: k_pre_deriv4_pairs<4, 2><<<grid2, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw, patw, ls, d_block); break;
            default: k_pre_deriv4_pairs<8, 2><<<grid2, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw, patw, ls, d_block); break;
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return final_sums(grid2 * (kT4 / 32));
    }
    const int grid = (d.Pp + kT4 / d.C - 1) / (kT4 / d.C);
    if (variant == 3) {
        // the staged-matrix walk
        switch (d.C) {
            case 1: k_pre_deriv4s<Real, 1><<<grid, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw, patw, ls, d_block); break;
            case 2: k_pre_deriv4s<Real, 2><<<grid, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw, patw, ls, d_block); break;
            case 4: k_pre_deriv4s<Real, 4><<<grid, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw, patw, ls, d_block); break;
            default: k_pre_deriv4s<Real, 8><<<grid, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw, patw, ls, d_block); break;
        }
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        return final_sums(fused_blocks(d));
    }
    bool shared_d = true;             // one derivative matrix for every branch
    for (int k = 1; k < nops; ++k)
        shared_d = shared_d && h_ops[k].dmat == h_ops[0].dmat && h_ops[k].dpad == h_ops[0].dpad;
    // Every pair shares its two matrices: FP32 holds them in registers (and
    // loads the derivative matrix per op: both in registers would spill).
    bool mats = sizeof(Real) == 4;
    for (int k = 0; k < nops; ++k)
        if ((h_ops[k].kind & kPairFirst) && !(h_ops[k].kind & kPairMats)) mats = false;
    if (mats) shared_d = false;
#define PD2_(CC, SD)                                                                        \
    (mats ? (k_pre_deriv4<Real, CC, SD, true><<<grid, kT4, 0, s>>>(prm, nops, d.P, d.Pp, catw,  \
                                                                  patw, ls, d_block), 0)     \
          : (k_pre_deriv4<Real, CC, SD, false><<<grid, kT4, 0, s>>>(prm, nops, d.P, d.Pp,    \
                                                                   catw, patw, ls, d_block), 0))
#define PD_(CC) (shared_d ? PD2_(CC, true) : PD2_(CC, false))
    switch (d.C) {
        case 1: PD_(1); break;
        case 2: PD_(2); break;
        case 4: PD_(4); break;
        default: PD_(8); break;
    }
#undef PD2_
#undef PD_
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return final_sums(fused_blocks(d));
}

}  // namespace

// Lists longer than kFusedOps run as consecutive launches, cut between
// sibling pairs: a launch boundary orders every write of one launch before
// every read of the next, so the cut changes only the launch count.  The
// scratch d_block is reused by each launch in stream order.
template <typename Real>
cudaError_t launch_pre_deriv4(const PreDerivOp* h_ops, int nops, const Dims& d,
                              const double* catw, const double* patw, int ls, double* d_block,
                              double* d_sums, cudaStream_t s, int variant) {
    if (nops == 0) return cudaSuccess;
    if (!fused_supported(d, nops)) return cudaErrorInvalidValue;
    for (int o0 = 0; o0 < nops;) {
        int e = std::min(nops, o0 + kFusedOps);
        if (e < nops && (h_ops[e - 1].kind & kPairFirst)) --e;   // keep the pair together
        const cudaError_t r = pre_deriv4_chunk<Real>(h_ops + o0, e - o0, d, catw, patw, ls,
                                                     d_block, d_sums + o0, nops, s, variant);
        if (r != cudaSuccess) return r;
        o0 = e;
    }
    return cudaSuccess;
}

template cudaError_t launch_pre_deriv4<float>(const PreDerivOp*, int, const Dims&, const double*,
                                              const double*, int, double*, double*, cudaStream_t,
                                              int);
template cudaError_t launch_pre_deriv4<double>(const PreDerivOp*, int, const Dims&, const double*,
                                               const double*, int, double*, double*,
                                               cudaStream_t, int);

}  // namespace b200
