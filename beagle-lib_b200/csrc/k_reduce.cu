// Pattern reductions: root and edge log-likelihoods, edge derivatives and
// scale-factor accumulation.  All sums that leave the device are FP64 and
// deterministic: fixed 128-thread blocks reduce by warp shuffles and shared
// memory into per-block partial sums, and a second pass (one CTA per output)
// adds the partials in a fixed order.
#include <cstdlib>
#include "b200_kernels.h"
#include "b200_vec.cuh"

namespace b200 {

__device__ int b200_bulk_status;   // nonzero: a bulk-copy kernel gave up waiting

namespace {

constexpr int kRB = 128;   // reduction block size (patterns per block)

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of v over the block (kRB threads); result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kRB / 32; ++w) t += sh[w];
    return t;
}

// Sum of v over a block of N threads; result valid in thread 0.
template <int N>
__device__ __forceinline__ double block_sum_n(double v, double* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < N / 32; ++w) t += sh[w];
    return t;
}

// out[k] = sum over the nblk partials in[k * nblk + b]; one CTA per output,
// each thread adding a fixed strided subset, then a fixed-order block sum.
__global__ void k_final_sum(const double* __restrict__ in, int nblk, int nout, double* out) {
    __shared__ double sh[kRB / 32];
    const int k = blockIdx.x;
    double v = 0;
    for (int b = threadIdx.x; b < nblk; b += kRB) v += in[(size_t)k * nblk + b];
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) out[k] = t;
    (void)nout;
}

// Site value of sum_c w_c sum_i pi_i x[p][c][i] for a partials buffer; the
// category sum runs first, as in CPU/BeagleCPUImpl.hpp:2646-2673.
template <typename Real>
__device__ __forceinline__ double integrate_site(const Real* x, const double* catw,
                                                 const double* freqs, int S, int Sg, int C,
                                                 int p) {
    const Real* xp = x + (size_t)p * C * Sg;
    double sum = 0;
    for (int i = 0; i < S; ++i) {
        double integ = 0;
        for (int c = 0; c < C; ++c) integ += (double)xp[c * Sg + i] * catw[c];
        sum += freqs[i] * integ;
    }
    return sum;
}

// Root log-likelihood of patterns [p_begin, p_end) with LP lanes per pattern
// (a power of two <= 32).  A pattern's C x Sg values are C * Sg / 4
// four-state groups, contiguous in the [pattern][category][state] layout;
// lane l of the pattern's group adds freqs[i] * (w_c * x[c][i]) over groups
// l, l + LP, ..., and a shuffle sum inside the lane group gives the site
// value.  The reference sums over categories first
// (CPU/BeagleCPUImpl.hpp:2646-2673); the terms are the same, added in
// another order, so the site values agree to FP64 rounding.  Several lanes
// per pattern keep a few thousand patterns of 61 states on every SM.
template <typename Real, int LP>
__global__ void __launch_bounds__(kRB)
k_root_lnl(const Real* __restrict__ root, const double* __restrict__ catw,
           const double* __restrict__ freqs, const double* __restrict__ cum,
           const double* __restrict__ patw, int S, int Sg, int C, int p_begin, int p_end,
           double* site, double* block) {
    __shared__ double sh[kRB / 32];
    const int lane = threadIdx.x % LP;
    const int p = p_begin + blockIdx.x * (kRB / LP) + threadIdx.x / LP;
    const int G = Sg / 4;
    double acc = 0;
    if (p < p_end) {
        const Real* xp = root + (size_t)p * C * Sg;
        for (int t = lane; t < C * G; t += LP) {
            const int c = t / G, i0 = 4 * (t - c * G);
            Real x[4];
            ld4(xp + 4 * (size_t)t, x);
            const double w = catw[c];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (i0 + q < S) acc += freqs[i0 + q] * (w * (double)x[q]);
        }
    }
#pragma unroll
    for (int o = LP / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    double v = 0;
    if (lane == 0 && p < p_end) {
        double l = log(acc);
        if (cum) l += cum[p];
        site[p] = l;
        v = l * patw[p];
    }
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) block[blockIdx.x] = t;
}

// Edge log-likelihood with optional derivative sums
// (CPU/BeagleCPUImpl.hpp:3209-3322, 3753-3994): with
// L = sum_c w_c sum_i pi_i parent[c,p,i] (M . child)[c,p,i] for M = P, P', P'',
// site lnL = log L + cumulative, d1 = L'/L, d2 = L''/L - d1^2.
template <typename Real>
__device__ __forceinline__ double edge_integrate(const Real* par, const void* child, bool states,
                                                 const Real* M, double pad,
                                                 const double* catw, const double* freqs,
                                                 int S, int Sg, int C, int p) {
    const Real* pp = par + (size_t)p * C * Sg;
    double tot = 0;
    if (states) {
        const int s = static_cast<const int*>(child)[p];
        for (int c = 0; c < C; ++c) {
            double acc = 0;
            for (int i = 0; i < S; ++i) {
                const double m = (s < S) ? (double)M[(size_t)c * Sg * Sg + i * Sg + s] : pad;
                acc += freqs[i] * m * (double)pp[c * Sg + i];
            }
            tot += catw[c] * acc;
        }
    } else {
        const Real* cp = static_cast<const Real*>(child) + (size_t)p * C * Sg;
        for (int c = 0; c < C; ++c) {
            double acc = 0;
            for (int i = 0; i < S; ++i) {
                double y = 0;
                const Real* row = M + (size_t)c * Sg * Sg + i * Sg;
                for (int j = 0; j < S; ++j) y += (double)row[j] * (double)cp[c * Sg + j];
                acc += freqs[i] * y * (double)pp[c * Sg + i];
            }
            tot += catw[c] * acc;
        }
    }
    return tot;
}

template <typename Real>
__global__ void __launch_bounds__(kRB)
k_edge_lnl(const Real* __restrict__ par, const void* child, int states, const Real* pm,
           double ppad, const Real* d1m, double d1pad, const Real* d2m, double d2pad,
           const double* __restrict__ catw, const double* __restrict__ freqs,
           const double* __restrict__ cum, const double* __restrict__ patw, int S, int Sg,
           int C, int p_begin, int p_end, double* site, double* site1, double* site2,
           double* block) {
    __shared__ double sh[kRB / 32];
    const int p = p_begin + blockIdx.x * kRB + threadIdx.x;
    double v0 = 0, v1 = 0, v2 = 0;
    if (p < p_end) {
        const double L = edge_integrate(par, child, states, pm, ppad, catw, freqs, S, Sg, C, p);
        double l = log(L);
        if (cum) l += cum[p];
        site[p] = l;
        v0 = l * patw[p];
        if (d1m) {
            const double g1 =
                edge_integrate(par, child, states, d1m, d1pad, catw, freqs, S, Sg, C, p) / L;
            site1[p] = g1;
            v1 = g1 * patw[p];
            if (d2m) {
                const double g2 =
                    edge_integrate(par, child, states, d2m, d2pad, catw, freqs, S, Sg, C, p) / L -
                    g1 * g1;
                site2[p] = g2;
                v2 = g2 * patw[p];
            }
        }
    }
    const int nb = gridDim.x;
    double t = block_sum(v0, sh);
    if (threadIdx.x == 0) block[blockIdx.x] = t;
    t = block_sum(v1, sh);
    if (threadIdx.x == 0) block[nb + blockIdx.x] = t;
    t = block_sum(v2, sh);
    if (threadIdx.x == 0) block[2 * nb + blockIdx.x] = t;
}

// Edge derivative of one branch (blockIdx.y) over a block of patterns
// (CPU/BeagleCPUImpl.hpp:1940-2083, :2086-2119, :2240-2285):
//   num = sum_c w_c sum_k pre[c,p,k] (D_c . post)[c,p,k],
//   den = sum_c w_c sum_k pre[c,p,k] post[c,p,k],  d = num / den.
// A compact post operand is a one-hot column (D[k][s], pre[s]); the missing
// state is an all-ones partial (D's pad value, sum_k pre[k]).
// Per-category terms are formed in Real, accumulated over categories in FP64.
template <typename Real>
__global__ void __launch_bounds__(kRB)
k_edge_deriv(const DerivDesc* __restrict__ desc, const double* __restrict__ catw,
             const double* __restrict__ patw, int S, int Sg, int C, int P, double* site,
             double* block) {
    __shared__ double sh[kRB / 32];
    const int b = blockIdx.y;
    const DerivDesc dd = desc[b];
    const int p = blockIdx.x * kRB + threadIdx.x;
    double d = 0;
    if (p < P) {
        const Real* pre = static_cast<const Real*>(dd.pre) + (size_t)p * C * Sg;
        const Real* D = static_cast<const Real*>(dd.dmat);
        double num = 0, den = 0;
        if (dd.post_is_states) {
            const int s = static_cast<const int*>(dd.post)[p];
            for (int c = 0; c < C; ++c) {
                Real n = 0, q = 0;
                for (int k = 0; k < S; ++k) {
                    const Real pk = pre[c * Sg + k];
                    const Real dk = (s < S) ? D[(size_t)c * Sg * Sg + k * Sg + s] : (Real)dd.dpad;
                    n += pk * dk;
                    if (s >= S || k == s) q += pk;
                }
                num += catw[c] * (double)n;
                den += catw[c] * (double)q;
            }
        } else {
            const Real* post = static_cast<const Real*>(dd.post) + (size_t)p * C * Sg;
            for (int c = 0; c < C; ++c) {
                Real n = 0, q = 0;
                const Real* Dc = D + (size_t)c * Sg * Sg;
                for (int k = 0; k < S; ++k) {
                    Real y = 0;
                    for (int j = 0; j < S; ++j) y += Dc[k * Sg + j] * post[c * Sg + j];
                    const Real pk = pre[c * Sg + k];
                    n += pk * y;
                    q += pk * post[c * Sg + k];
                }
                num += catw[c] * (double)n;
                den += catw[c] * (double)q;
            }
        }
        d = num / den;
        if (site) site[(size_t)b * P + p] = d;
    }
    const double w = (p < P) ? patw[p] : 0.0;
    const int nblk = gridDim.x;
    double t = block_sum(d * w, sh);
    if (threadIdx.x == 0) block[(size_t)b * nblk + blockIdx.x] = t;
    t = block_sum(d * d * w, sh);
    if (threadIdx.x == 0) block[(size_t)(gridDim.y + b) * nblk + blockIdx.x] = t;
}

// S = 4 specialisation of k_edge_deriv: one thread per (pattern, category)
// with 16-byte (FP32) / 32-byte (FP64) vector loads; the C threads of a
// pattern combine their weighted terms with shuffles.  A tile is kRB / C * PPT
// patterns (each thread covers PPT patterns kRB / C apart); a CTA walks ITER
// consecutive tiles of one branch (blockIdx.y), loading tile i + 1 while it
// computes tile i, and pays its two block reductions once at the end.  The
// category's 4x4 derivative matrix is held in registers throughout.
// d = sum_c w_c num_c / sum_c w_c den_c over the C lanes of one pattern, in
// the partials' precision (the FP64 path stays FP64); callers accumulate the
// weighted sums of d in FP64.
template <typename Real, int C>
__device__ __forceinline__ Real combine_categories(Real n, Real q, Real w) {
    Real num = w * n, den = w * q;
#pragma unroll
    for (int o = 1; o < C; o <<= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
    }
    return num / den;
}

template <typename Real, int PPT>
struct DerivRows4 {
    Real z[PPT][4];   // pre-order partials
    Real x[PPT][4];   // post-order partials
    int st[PPT];      // or tip states
};

template <typename Real, int C, int PPT>
__device__ __forceinline__ void deriv4_load(DerivRows4<Real, PPT>& r, const DerivDesc& dd,
                                            bool states, int p0, int P, int c) {
    constexpr int kSlots = kRB / C;
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        const int pc = min(p0 + j * kSlots, P - 1);
        ld4(static_cast<const Real*>(dd.pre) + ((size_t)pc * C + c) * 4, r.z[j]);
        if (states)
            r.st[j] = static_cast<const int*>(dd.post)[pc];
        else
            ld4(static_cast<const Real*>(dd.post) + ((size_t)pc * C + c) * 4, r.x[j]);
    }
}

// Derivative terms of one tile (this thread's PPT patterns p0 + j kRB / C):
// per-site value into site[b * P + p] when requested, weighted sums into s1, s2.
template <typename Real, int C, int PPT>
__device__ __forceinline__ void deriv4_tile(const DerivRows4<Real, PPT>& cur, const Real dm[16],
                                            Real w, const DerivDesc& dd, bool states, int p0,
                                            int P, const double* __restrict__ patw, int b,
                                            double* site, double& s1, double& s2) {
    constexpr int kSlots = kRB / C;
    const int c = threadIdx.x % C;
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        const int p = p0 + j * kSlots;
        Real n = 0, q = 0;
        if (states) {
            const int s = cur.st[j];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                Real dk = (Real)dd.dpad;
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (s == i) dk = dm[k * 4 + i];
                n += cur.z[j][k] * dk;
                q += (s >= 4 || k == s) ? cur.z[j][k] : Real(0);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const Real y = dm[k * 4] * cur.x[j][0] + dm[k * 4 + 1] * cur.x[j][1] +
                               dm[k * 4 + 2] * cur.x[j][2] + dm[k * 4 + 3] * cur.x[j][3];
                n += cur.z[j][k] * y;
                q += cur.z[j][k] * cur.x[j][k];
            }
        }
        const Real dr = combine_categories<Real, C>(n, q, w);
        if (c == 0 && p < P) {
            const double d = (double)dr;
            if (site) site[(size_t)b * P + p] = d;
            const double wp = patw[p];
            s1 += d * wp;
            s2 += d * d * wp;
        }
    }
}

template <typename Real, int C, int ITER, int PPT>
__global__ void __launch_bounds__(kRB)
k_edge_deriv4(const DerivDesc* __restrict__ desc, const double* __restrict__ catw,
              const double* __restrict__ patw, int P, double* site, double* block) {
    __shared__ double sh[kRB / 32];
    constexpr int kSlots = kRB / C;
    constexpr int kTile = kSlots * PPT;
    const int b = blockIdx.y;
    const int c = threadIdx.x % C;
    const int t0 = blockIdx.x * ITER;                  // first tile of this CTA
    const int ntiles = (P + kTile - 1) / kTile;
    const DerivDesc& dd = desc[b];
    const Real* D = static_cast<const Real*>(dd.dmat) + c * 16;
    Real dm[16];
#pragma unroll
    for (int k = 0; k < 4; ++k) ld4(D + 4 * k, dm + 4 * k);
    const Real w = (Real)catw[c];
    const bool states = dd.post_is_states;
    DerivRows4<Real, PPT> cur, nxt;
    deriv4_load<Real, C, PPT>(cur, dd, states, t0 * kTile + threadIdx.x / C, P, c);
    double s1 = 0, s2 = 0;
#pragma unroll 1
    for (int it = 0; it < ITER; ++it) {
        if (t0 + it >= ntiles) break;
        const int p0 = (t0 + it) * kTile + threadIdx.x / C;
        if (it + 1 < ITER && t0 + it + 1 < ntiles)
            deriv4_load<Real, C, PPT>(nxt, dd, states, p0 + kTile, P, c);
        deriv4_tile<Real, C, PPT>(cur, dm, w, dd, states, p0, P, patw, b, site, s1, s2);
        cur = nxt;
    }
    const int nblk = gridDim.x;
    double t = block_sum(s1, sh);
    if (threadIdx.x == 0) block[(size_t)b * nblk + blockIdx.x] = t;
    t = block_sum(s2, sh);
    if (threadIdx.x == 0) block[(size_t)(gridDim.y + b) * nblk + blockIdx.x] = t;
}

// ---------------------------------------------------- S = 4, bulk-copy stream
// The derivative pass is a pure stream: per branch it reads the pre-order and
// the post-order partials (or tip states) once.  This variant keeps that
// stream in flight with bulk asynchronous copies.  One CTA per SM walks work
// items (branch, chunk of 16 KB per operand: 256 patterns of 4 FP32
// categories) in a fixed order; a chunk of a
// partials buffer is contiguous in the [pattern][category][state] layout, so
// each operand is one cp.async.bulk into a shared-memory stage, completed on
// the stage's mbarrier.  Thread 0 keeps kBulkStages - 1 items in flight
// ahead of the one the CTA computes.  Every item writes its own pair of block
// partial sums (branch, chunk), so the final sums do not depend on which CTA
// took which item.  Waits are bounded (b200_bulk_status on time-out).
constexpr int kBulkStageBytes = 16384;   // per operand and stage
constexpr int kBulkStages = 3;
constexpr int kBulkThreads = 512;
constexpr long long kBulkWaitCycles = 2000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bulk_bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void bulk_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// dst (shared) <- src (global), `bytes` a multiple of 16, both 16-byte aligned.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// A wait bounded below the default polls with the non-blocking test_wait:
// try_wait may suspend the thread until the phase completes, which would
// outlast a short bound.
__device__ __forceinline__ void bulk_wait(uint64_t* bar, uint32_t parity, bool& failed,
                                          long long limit = kBulkWaitCycles) {
    if (failed) return;
    const bool poll = limit < kBulkWaitCycles;
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        if (poll)
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(ok)
                : "r"(smem_addr(bar)), "r"(parity)
                : "memory");
        else
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(ok)
                : "r"(smem_addr(bar)), "r"(parity)
                : "memory");
        if (ok) return;
        if (clock64() - t0 > limit) {
            failed = true;
            atomicExch(&b200_bulk_status, 1);
            return;
        }
    }
}

// Issue the copies of work item `item` into stage `st` (thread 0 only).
template <typename Real, int C>
constexpr int bulk_tile() { return kBulkStageBytes / (C * 4 * (int)sizeof(Real)); }

template <typename Real, int C>
__device__ __forceinline__ void bulk_issue(const DerivDesc* desc, int item, int nchunks, int Pp,
                                           unsigned char* stage_pre, unsigned char* stage_post,
                                           uint64_t* bar) {
    const int b = item / nchunks, q = item - b * nchunks;
    const DerivDesc& dd = desc[b];
    const int p0 = q * bulk_tile<Real, C>();
    const int rows = min(bulk_tile<Real, C>(), Pp - p0);
    const uint32_t row_bytes = (uint32_t)(C * 4 * sizeof(Real));
    const uint32_t pre_bytes = rows * row_bytes;
    const uint32_t post_bytes = dd.post_is_states ? (uint32_t)(((rows * 4) + 15) & ~15)
                                                  : pre_bytes;
    bulk_expect(bar, pre_bytes + post_bytes);
    bulk_copy(stage_pre, static_cast<const unsigned char*>(dd.pre) + (size_t)p0 * row_bytes,
              pre_bytes, bar);
    if (dd.post_is_states)
        bulk_copy(stage_post, static_cast<const int*>(dd.post) + p0, post_bytes, bar);
    else
        bulk_copy(stage_post, static_cast<const unsigned char*>(dd.post) + (size_t)p0 * row_bytes,
                  post_bytes, bar);
}

template <typename Real, int C>
__global__ void __launch_bounds__(kBulkThreads)
k_edge_deriv4_bulk(const DerivDesc* __restrict__ desc, const double* __restrict__ catw,
                   const double* __restrict__ patw, int P, int Pp, int nb, double* site,
                   double* block, long long wait_cycles) {
    constexpr int kTile = bulk_tile<Real, C>();
    constexpr size_t kStageBytes = kBulkStageBytes;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* st_pre = smem_raw;                                   // [stages][kStageBytes]
    unsigned char* st_post = smem_raw + kBulkStages * kStageBytes;      // [stages][kStageBytes]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + 2 * kBulkStages * kStageBytes);
    __shared__ double sh[kBulkThreads / 32];
    const int nchunks = (Pp + kTile - 1) / kTile;
    const int nitems = nb * nchunks;
    const int c = threadIdx.x % C;
    constexpr int kSlots = kBulkThreads / C;          // patterns per pass over the chunk
    constexpr int kPasses = kTile / kSlots;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kBulkStages; ++s) bulk_bar_init(&bars[s]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // Copies issued into each stage (thread 0's count; stage s's k-th copy
    // completes the barrier's phase k, of parity k & 1).
    int issued[kBulkStages] = {};
    // Prologue: the first kBulkStages items of this CTA.
    if (threadIdx.x == 0) {
        for (int s = 0; s < kBulkStages; ++s) {
            const int item = blockIdx.x + s * gridDim.x;
            if (item < nitems) {
                bulk_issue<Real, C>(desc, item, nchunks, Pp, st_pre + s * kStageBytes,
                                    st_post + s * kStageBytes, &bars[s]);
                ++issued[s];
            }
        }
    }
    bool failed = false;
    uint32_t phase[kBulkStages] = {};
    int s = 0;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int b = item / nchunks, q = item - b * nchunks;
        const DerivDesc& dd = desc[b];
        bulk_wait(&bars[s], phase[s], failed, wait_cycles);
        phase[s] ^= 1u;
        const Real* pre = reinterpret_cast<const Real*>(st_pre + s * kStageBytes);
        const Real* post = reinterpret_cast<const Real*>(st_post + s * kStageBytes);
        const int* tip = reinterpret_cast<const int*>(st_post + s * kStageBytes);
        const bool states = dd.post_is_states;
        const Real* D = static_cast<const Real*>(dd.dmat) + c * 16;
        Real dm[16];
#pragma unroll
        for (int k = 0; k < 4; ++k) ldg4(D + 4 * k, dm + 4 * k);
        const Real w = (Real)catw[c];
        double s1 = 0, s2 = 0;
#pragma unroll
        for (int j = 0; j < kPasses; ++j) {
            const int r = j * kSlots + threadIdx.x / C;     // row in the chunk
            const int p = q * kTile + r;
            Real z[4], x[4];
            ld4(pre + ((size_t)r * C + c) * 4, z);
            Real n = 0, qd = 0;
            if (states) {
                const int st = p < Pp ? tip[r] : 4;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    Real dk = (Real)dd.dpad;
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (st == i) dk = dm[k * 4 + i];
                    n += z[k] * dk;
                    qd += (st >= 4 || k == st) ? z[k] : Real(0);
                }
            } else {
                ld4(post + ((size_t)r * C + c) * 4, x);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const Real y = dm[k * 4] * x[0] + dm[k * 4 + 1] * x[1] + dm[k * 4 + 2] * x[2] +
                                   dm[k * 4 + 3] * x[3];
                    n += z[k] * y;
                    qd += z[k] * x[k];
                }
            }
            const Real dr = combine_categories<Real, C>(n, qd, w);
            if (c == 0 && p < P) {
                const double d = (double)dr;
                if (site) site[(size_t)b * P + p] = d;
                const double wp = patw[p];
                s1 += d * wp;
                s2 += d * d * wp;
            }
        }
        // block_sum's barriers also mark stage s as consumed by every thread
        double t = block_sum_n<kBulkThreads>(s1, sh);
        if (threadIdx.x == 0) block[(size_t)b * nchunks + q] = t;
        t = block_sum_n<kBulkThreads>(s2, sh);
        if (threadIdx.x == 0) {
            block[(size_t)(nb + b) * nchunks + q] = t;
            const int next = item + kBulkStages * gridDim.x;
            if (next < nitems && !failed) {
                // every thread's reads of stage s are done (block_sum's barriers)
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                bulk_issue<Real, C>(desc, next, nchunks, Pp, st_pre + s * kStageBytes,
                                    st_post + s * kStageBytes, &bars[s]);
                ++issued[s];
            }
        }
        s = (s + 1) % kBulkStages;
    }
    // After a time-out, copies may still be in flight into this CTA's shared
    // memory: wait (with the full bound, whatever wait_cycles was) until the
    // phase of the last copy issued into each stage has completed, before the
    // CTA exits.  A completed phase returns at once.
    if (failed && threadIdx.x == 0) {
        for (int k = 0; k < kBulkStages; ++k) {
            if (issued[k] == 0) continue;
            bool again = false;
            bulk_wait(&bars[k], (uint32_t)((issued[k] - 1) & 1), again);
        }
    }
}

// BEAGLE_B200_WAIT_CYCLES: the bound, in clock cycles, of the bulk-copy
// derivative's waits on its stages (default 2e9, about one second).  Lower
// values exist so that tests can make a wait run out on purpose and check
// that the time-out is reported; the wait for copies still in flight before
// a CTA exits always keeps the full bound.
long long bulk_wait_cycles() {
    const char* v = std::getenv("BEAGLE_B200_WAIT_CYCLES");
    if (!v || !*v) return kBulkWaitCycles;
    const long long x = std::atoll(v);
    return x > 0 ? x : kBulkWaitCycles;
}

template <typename Real, int C>
cudaError_t run_deriv4_bulk(const DerivDesc* desc, int nb, const double* catw,
                            const double* patw, const Dims& d, double* site, double* block,
                            cudaStream_t s) {
    const size_t smem = 2 * kBulkStages * (size_t)kBulkStageBytes + kBulkStages * sizeof(uint64_t);
    auto kern = k_edge_deriv4_bulk<Real, C>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBulkThreads, smem);
    if (e != cudaSuccess) return e;
    constexpr int kTile = bulk_tile<Real, C>();
    const int nitems = nb * ((d.Pp + kTile - 1) / kTile);
    const int slots = sms * (per_sm > 0 ? per_sm : 1);
    const int grid = nitems < slots ? nitems : slots;
    kern<<<grid, kBulkThreads, smem, s>>>(desc, catw, patw, d.P, d.Pp, nb, site, block,
                                          bulk_wait_cycles());
    return cudaGetLastError();
}

// ------------------------------------------------- batched reductions
// One launch for several instances (b200_batch.cpp).  CTA x belongs to the
// segment whose first_cta is the largest one <= x.
template <typename Seg>
__device__ __forceinline__ int find_seg(const Seg* segs, int nseg, int x) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].first_cta <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// S = 4 edge derivatives of several instances with the same C: CTA (segment,
// branch b, block k) covers the 2 kRB / C patterns of tile k (two per thread).
template <typename Real, int C>
__global__ void __launch_bounds__(kRB)
k_deriv4_batch(const DerivSeg* __restrict__ segs, int nseg) {
    __shared__ double sh[kRB / 32];
    __shared__ int s_seg;
    constexpr int PPT = 2;
    constexpr int kTile = kRB / C * PPT;
    if (threadIdx.x == 0) s_seg = find_seg(segs, nseg, blockIdx.x);
    __syncthreads();
    const DerivSeg sg = segs[s_seg];
    const int local = blockIdx.x - sg.first_cta;
    const int b = local / sg.nblk, k = local - b * sg.nblk;
    const int c = threadIdx.x % C;
    const DerivDesc& dd = sg.desc[b];
    const Real* D = static_cast<const Real*>(dd.dmat) + c * 16;
    Real dm[16];
#pragma unroll
    for (int q = 0; q < 4; ++q) ld4(D + 4 * q, dm + 4 * q);
    const Real w = (Real)sg.catw[c];
    const bool states = dd.post_is_states;
    const int p0 = k * kTile + threadIdx.x / C;
    DerivRows4<Real, PPT> cur;
    deriv4_load<Real, C, PPT>(cur, dd, states, p0, sg.P, c);
    double s1 = 0, s2 = 0;
    deriv4_tile<Real, C, PPT>(cur, dm, w, dd, states, p0, sg.P, sg.patw, b, nullptr, s1, s2);
    double t = block_sum(s1, sh);
    if (threadIdx.x == 0) sg.block[(size_t)b * sg.nblk + k] = t;
    t = block_sum(s2, sh);
    if (threadIdx.x == 0) sg.block[(size_t)(sg.nb + b) * sg.nblk + k] = t;
}

// Root log-likelihoods of several instances (any state count): CTA (segment,
// block k) covers patterns [k kRB, (k + 1) kRB).
template <typename Real>
__global__ void __launch_bounds__(kRB)
k_root_batch(const RootSeg* __restrict__ segs, int nseg) {
    __shared__ double sh[kRB / 32];
    __shared__ int s_seg;
    if (threadIdx.x == 0) s_seg = find_seg(segs, nseg, blockIdx.x);
    __syncthreads();
    const RootSeg sg = segs[s_seg];
    const int k = blockIdx.x - sg.first_cta;
    const int p = k * kRB + threadIdx.x;
    double v = 0;
    if (p < sg.P) {
        double l = log(integrate_site(static_cast<const Real*>(sg.root), sg.catw, sg.freqs, sg.S,
                                      sg.Sg, sg.C, p));
        if (sg.cum) l += sg.cum[p];
        sg.site[p] = l;
        v = l * sg.patw[p];
    }
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) sg.block[k] = t;
}

// cumulative[p] = (reset ? 0 : cumulative[p]) + sum_i f(scale[idx_i][p]) for
// several instances; 256 patterns per CTA.
__global__ void k_accumulate_batch(const AccSeg* __restrict__ segs, int nseg) {
    __shared__ int s_seg;
    if (threadIdx.x == 0) s_seg = find_seg(segs, nseg, blockIdx.x);
    __syncthreads();
    const AccSeg sg = segs[s_seg];
    const int p = (blockIdx.x - sg.first_cta) * blockDim.x + threadIdx.x;
    if (p >= sg.P) return;
    double acc = sg.reset ? 0.0 : sg.cum[p];
    if (sg.log_scalers) {
#pragma unroll 8
        for (int i = 0; i < sg.n; ++i) acc += sg.pool[(size_t)__ldg(sg.idx + i) * sg.Pp + p];
    } else {
#pragma unroll 8
        for (int i = 0; i < sg.n; ++i) acc += log(sg.pool[(size_t)__ldg(sg.idx + i) * sg.Pp + p]);
    }
    sg.cum[p] = acc;
}

// Final sums of several instances' block partials: one CTA per output.
__global__ void k_final_batch(const FinalSeg* __restrict__ segs, int nseg) {
    __shared__ double sh[kRB / 32];
    __shared__ int s_seg;
    if (threadIdx.x == 0) {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (segs[mid].first_out <= (int)blockIdx.x) lo = mid;
            else hi = mid - 1;
        }
        s_seg = lo;
    }
    __syncthreads();
    const FinalSeg sg = segs[s_seg];
    const int k = blockIdx.x - sg.first_out;
    double v = 0;
    for (int b = threadIdx.x; b < sg.nblk; b += kRB) v += sg.block[(size_t)k * sg.nblk + b];
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) sg.out[k] = t;
}

__global__ void k_accumulate_scale(double* cum, const double* __restrict__ pool,
                                   const int* __restrict__ idx, int n, int Pp, int p_begin,
                                   int p_end, double sign, int log_scalers) {
    const int p = p_begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= p_end) return;
    // eight independent loads in flight per thread, added in buffer order
    double acc = 0;
    if (log_scalers) {
#pragma unroll 8
        for (int i = 0; i < n; ++i) acc += pool[(size_t)__ldg(idx + i) * Pp + p];
    } else {
#pragma unroll 8
        for (int i = 0; i < n; ++i) acc += log(pool[(size_t)__ldg(idx + i) * Pp + p]);
    }
    cum[p] += sign * acc;
}

}  // namespace

int reduction_blocks(int Pp) { return (Pp + kRB - 1) / kRB; }

// Lanes per pattern of the root reduction: enough that a lane adds at most
// 4 of a pattern's C * Sg / 4 four-state groups (1 for 4 states and up to 4
// categories, 16 for 61 states and 4 categories), at most 32.
int root_lanes(const Dims& d) {
    const int items = d.C * (d.Sg / 4);
    int lp = 1;
    while (lp < 32 && lp * 4 < items) lp <<= 1;
    return lp;
}

int root_blocks(const Dims& d, int n, bool wide) {
    const int ppb = kRB / (wide ? root_lanes(d) : 1);
    return (n + ppb - 1) / ppb;
}

template <typename Real>
cudaError_t launch_root_lnl(const void* root, const double* catw, const double* freqs,
                            const double* cum, const double* patw, const Dims& d,
                            double* d_site, double* d_block, double* d_out, cudaStream_t s,
                            bool wide) {
    return launch_root_lnl_range<Real>(root, catw, freqs, cum, patw, d, 0, d.P, d_site, d_block,
                                       d_out, s, wide);
}

template <typename Real>
cudaError_t launch_root_lnl_range(const void* root, const double* catw, const double* freqs,
                                  const double* cum, const double* patw, const Dims& d,
                                  int p_begin, int p_end, double* d_site, double* d_block,
                                  double* d_out, cudaStream_t s, bool wide) {
    const int nblk = root_blocks(d, p_end - p_begin, wide);
    if (nblk == 0) return cudaMemsetAsync(d_out, 0, sizeof(double), s);
    const Real* r = static_cast<const Real*>(root);
#define RL_(LP)                                                                            \
    k_root_lnl<Real, LP><<<nblk, kRB, 0, s>>>(r, catw, freqs, cum, patw, d.S, d.Sg, d.C,  \
                                              p_begin, p_end, d_site, d_block)
    switch (wide ? root_lanes(d) : 1) {
        case 1: RL_(1); break;
        case 2: RL_(2); break;
        case 4: RL_(4); break;
        case 8: RL_(8); break;
        case 16: RL_(16); break;
        default: RL_(32); break;
    }
#undef RL_
    k_final_sum<<<1, kRB, 0, s>>>(d_block, nblk, 1, d_out);
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_edge_lnl(const void* parent, const void* child, int child_is_states,
                            const void* pmat, double ppad, const void* d1mat, double d1pad,
                            const void* d2mat, double d2pad, const double* catw,
                            const double* freqs, const double* cum, const double* patw,
                            const Dims& d, double* d_site, double* d_site1, double* d_site2,
                            double* d_block, double* d_out, cudaStream_t s) {
    return launch_edge_lnl_range<Real>(parent, child, child_is_states, pmat, ppad, d1mat, d1pad,
                                       d2mat, d2pad, catw, freqs, cum, patw, d, 0, d.P, d_site,
                                       d_site1, d_site2, d_block, d_out, s);
}

template <typename Real>
cudaError_t launch_edge_lnl_range(const void* parent, const void* child, int child_is_states,
                                  const void* pmat, double ppad, const void* d1mat, double d1pad,
                                  const void* d2mat, double d2pad, const double* catw,
                                  const double* freqs, const double* cum, const double* patw,
                                  const Dims& d, int p_begin, int p_end, double* d_site,
                                  double* d_site1, double* d_site2, double* d_block,
                                  double* d_out, cudaStream_t s) {
    const int nblk = reduction_blocks(p_end - p_begin);
    if (nblk == 0) return cudaMemsetAsync(d_out, 0, 3 * sizeof(double), s);
    k_edge_lnl<Real><<<nblk, kRB, 0, s>>>(
        static_cast<const Real*>(parent), child, child_is_states, static_cast<const Real*>(pmat),
        ppad, static_cast<const Real*>(d1mat), d1pad, static_cast<const Real*>(d2mat), d2pad,
        catw, freqs, cum, patw, d.S, d.Sg, d.C, p_begin, p_end, d_site, d_site1, d_site2,
        d_block);
    k_final_sum<<<3, kRB, 0, s>>>(d_block, nblk, 3, d_out);
    return cudaGetLastError();
}

namespace {

bool deriv4_shape(const Dims& d) {
    return d.S == 4 && d.Sg == 4 && (d.C == 1 || d.C == 2 || d.C == 4 || d.C == 8);
}

// Variant v of the S = 4 derivative kernel: (patterns per thread, tiles per
// CTA) = (1,1) (2,1) (4,1) (8,1) (2,8) (4,4).
struct Deriv4Shape {
    int ppt, iter;
};
Deriv4Shape deriv4_shape_of(int v) {
    static const Deriv4Shape kShapes[] = {{1, 1}, {2, 1}, {4, 1}, {8, 1}, {2, 8}, {4, 4}};
    return kShapes[v < 0 ? 0 : v > 5 ? 5 : v];
}

template <typename Real, int C>
void run_deriv4(Deriv4Shape sh, dim3 grid, cudaStream_t s, const DerivDesc* desc,
                const double* catw, const double* patw, int P, double* site, double* block) {
#define D4_(PPT, IT) k_edge_deriv4<Real, C, IT, PPT><<<grid, kRB, 0, s>>>(desc, catw, patw, P, site, block)
    if (sh.iter == 8) D4_(2, 8);
    else if (sh.iter == 4) D4_(4, 4);
    else if (sh.ppt == 1) D4_(1, 1);
    else if (sh.ppt == 2) D4_(2, 1);
    else if (sh.ppt == 4) D4_(4, 1);
    else D4_(8, 1);
#undef D4_
}

}  // namespace

// Variants 0-5: k_edge_deriv4 shapes (deriv4_shape_of); 6: the bulk-copy stream.
int deriv4_variants(const Dims& d) { return deriv4_shape(d) ? 7 : 1; }

template <typename Real>
cudaError_t launch_edge_derivatives(const DerivDesc* desc, int nb, const double* catw,
                                    const double* patw, const Dims& d, double* d_site,
                                    double* d_block, double* d_sums, cudaStream_t s,
                                    int variant) {
    if (nb == 0) return cudaSuccess;
    int nblk = reduction_blocks(d.P);
    if (deriv4_shape(d) && variant == 6) {
        cudaError_t e;
        int tile;
        switch (d.C) {
            case 1: e = run_deriv4_bulk<Real, 1>(desc, nb, catw, patw, d, d_site, d_block, s); tile = bulk_tile<Real, 1>(); break;
            case 2: e = run_deriv4_bulk<Real, 2>(desc, nb, catw, patw, d, d_site, d_block, s); tile = bulk_tile<Real, 2>(); break;
            case 4: e = run_deriv4_bulk<Real, 4>(desc, nb, catw, patw, d, d_site, d_block, s); tile = bulk_tile<Real, 4>(); break;
            default: e = run_deriv4_bulk<Real, 8>(desc, nb, catw, patw, d, d_site, d_block, s); tile = bulk_tile<Real, 8>(); break;
        }
        if (e != cudaSuccess) return e;
        nblk = (d.Pp + tile - 1) / tile;
    } else if (deriv4_shape(d)) {
        if (variant < 0) variant = d.P >= 32768 ? 2 : 0;
        const Deriv4Shape sh = deriv4_shape_of(variant);
        const int tile = kRB / d.C * sh.ppt;
        const int ntiles = (d.P + tile - 1) / tile;
        nblk = (ntiles + sh.iter - 1) / sh.iter;
        dim3 grid(nblk, nb);
        switch (d.C) {
            case 1: run_deriv4<Real, 1>(sh, grid, s, desc, catw, patw, d.P, d_site, d_block); break;
            case 2: run_deriv4<Real, 2>(sh, grid, s, desc, catw, patw, d.P, d_site, d_block); break;
            case 4: run_deriv4<Real, 4>(sh, grid, s, desc, catw, patw, d.P, d_site, d_block); break;
            default: run_deriv4<Real, 8>(sh, grid, s, desc, catw, patw, d.P, d_site, d_block); break;
        }
    } else {
        dim3 grid(nblk, nb);
        k_edge_deriv<Real><<<grid, kRB, 0, s>>>(desc, catw, patw, d.S, d.Sg, d.C, d.P, d_site,
                                                d_block);
    }
    k_final_sum<<<2 * nb, kRB, 0, s>>>(d_block, nblk, 2 * nb, d_sums);
    return cudaGetLastError();
}

cudaError_t bulk_status_async(int* pinned_dst, cudaStream_t s) {
    return cudaMemcpyFromSymbolAsync(pinned_dst, b200_bulk_status, sizeof(int), 0,
                                     cudaMemcpyDeviceToHost, s);
}

cudaError_t bulk_raise_status(cudaStream_t s) {
    static const int one = 1;
    return cudaMemcpyToSymbolAsync(b200_bulk_status, &one, sizeof(int), 0,
                                   cudaMemcpyHostToDevice, s);
}

cudaError_t bulk_clear_status(cudaStream_t s) {
    static const int zero = 0;
    return cudaMemcpyToSymbolAsync(b200_bulk_status, &zero, sizeof(int), 0,
                                   cudaMemcpyHostToDevice, s);
}

cudaError_t launch_deriv_final(const double* d_block, int nblk, int nb, double* d_sums,
                               cudaStream_t s) {
    k_final_sum<<<2 * nb, kRB, 0, s>>>(d_block, nblk, 2 * nb, d_sums);
    return cudaGetLastError();
}

cudaError_t launch_final_sum(const double* d_block, int nblk, int nout, double* d_out,
                             cudaStream_t s) {
    k_final_sum<<<nout, kRB, 0, s>>>(d_block, nblk, nout, d_out);
    return cudaGetLastError();
}

cudaError_t launch_deriv_final_at(const double* d_block, int nblk, int nb, double* d_sums,
                                  double* d_sumsq, cudaStream_t s) {
    k_final_sum<<<nb, kRB, 0, s>>>(d_block, nblk, nb, d_sums);
    k_final_sum<<<nb, kRB, 0, s>>>(d_block + (size_t)nb * nblk, nblk, nb, d_sumsq);
    return cudaGetLastError();
}

// ---------------------------------------------------- cross products
// beagleCalculateCrossProductDerivative (CPU/BeagleCPUImpl.hpp:1865-1937,
// :2122-2237): for every listed branch b and pattern p,
//   den = sum_c w_c sum_k pre[c,p,k] post[c,p,k]
//   out[k][j] += W_p / den * sum_c fac[b][c] pre[c,p,k] post[c,p,j],
// fac[b][c] = w_c r_c t_b, a tip's post row one-hot (all ones when missing).
// CTA = a tile of TP patterns, looping over the branches: the tile's rows are
// staged in shared memory, the pre rows scaled by W_p / den * fac, and each
// thread keeps up to 16 of the S x S sums (S <= 64) in FP64, adding the
// tile's TP * C terms in the partials' precision.  block[q][tile] holds the
// tile sums; k_final_sum adds the tiles in a fixed order.
constexpr int kCrossThreads = 256;

template <typename Real>
__global__ void __launch_bounds__(kCrossThreads)
k_cross_products(const DerivDesc* __restrict__ desc, int nb, const double* __restrict__ catw,
                 const double* __restrict__ fac, const double* __restrict__ patw, int S, int Sg,
                 int C, int P, int TP, double* block) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* coef = reinterpret_cast<double*>(smem_raw);            // [TP]
    Real* a = reinterpret_cast<Real*>(coef + TP);                  // [TP * C][Sg]
    Real* x = a + (size_t)TP * C * Sg;                             // [TP * C][Sg]
    const int tid = threadIdx.x;
    const int tile = blockIdx.x, ntiles = gridDim.x;
    const int p0 = tile * TP;
    const int row = C * Sg, n = TP * row, SS = S * S;
    double acc[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) acc[r] = 0.0;
    for (int b = 0; b < nb; ++b) {
        const DerivDesc d = desc[b];
        __syncthreads();   // the previous branch's reads of a, x, coef are done
        const Real* pre = static_cast<const Real*>(d.pre) + (size_t)p0 * row;
        for (int e = tid; e < n; e += kCrossThreads) {
            const int p = p0 + e / row;
            const int i = e % Sg;
            Real pv = 0, xv = 0;
            if (p < P) {
                pv = pre[e];
                if (d.post_is_states) {
                    const int st = static_cast<const int*>(d.post)[p];
                    xv = (i < S && (st >= S || st == i)) ? Real(1) : Real(0);
                } else {
                    xv = static_cast<const Real*>(d.post)[(size_t)p0 * row + e];
                }
            }
            a[e] = pv;
            x[e] = xv;
        }
        __syncthreads();
        for (int pl = tid; pl < TP; pl += kCrossThreads) {
            const int p = p0 + pl;
            double den = 0;
            for (int c = 0; c < C; ++c) {
                double dc = 0;
                for (int k = 0; k < S; ++k)
                    dc += (double)a[(pl * C + c) * Sg + k] * (double)x[(pl * C + c) * Sg + k];
                den += catw[c] * dc;
            }
            coef[pl] = p < P ? patw[p] / den : 0.0;
        }
        __syncthreads();
        for (int e = tid; e < n; e += kCrossThreads) {
            const int pl = e / row, c = (e / Sg) % C;
            a[e] = (Real)((double)a[e] * coef[pl] * fac[(size_t)b * C + c]);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int q = tid + kCrossThreads * r;
            if (q < SS) {
                const int k = q / S, j = q - (q / S) * S;
                Real sum = 0;
                for (int pc = 0; pc < TP * C; ++pc) sum += a[pc * Sg + k] * x[pc * Sg + j];
                acc[r] += (double)sum;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const int q = tid + kCrossThreads * r;
        if (q < SS) block[(size_t)q * ntiles + tile] = acc[r];
    }
}

// Patterns per tile and tiles of a cross-product launch.
int cross_tile_patterns(const Dims& d, bool dbl) {
    const int elems = dbl ? 2048 : 4096;
    int tp = elems / (d.C * d.Sg);
    tp = tp < 1 ? 1 : tp > 128 ? 128 : tp;
    return tp;
}

template <typename Real>
cudaError_t launch_cross_products(const DerivDesc* d_desc, int nb, const double* catw,
                                  const double* fac, const double* patw, const Dims& d,
                                  double* d_block, double* d_out, cudaStream_t s) {
    if (nb == 0) return cudaSuccess;
    if (d.S > 64) return cudaErrorInvalidValue;
    const int tp = cross_tile_patterns(d, sizeof(Real) == 8);
    const int ntiles = (d.P + tp - 1) / tp;
    const size_t smem = sizeof(double) * tp + 2 * sizeof(Real) * (size_t)tp * d.C * d.Sg;
    k_cross_products<Real><<<ntiles, kCrossThreads, smem, s>>>(d_desc, nb, catw, fac, patw, d.S,
                                                               d.Sg, d.C, d.P, tp, d_block);
    const int SS = d.S * d.S;
    k_final_sum<<<SS, kRB, 0, s>>>(d_block, ntiles, SS, d_out);
    return cudaGetLastError();
}

template cudaError_t launch_cross_products<float>(const DerivDesc*, int, const double*,
                                                  const double*, const double*, const Dims&,
                                                  double*, double*, cudaStream_t);
template cudaError_t launch_cross_products<double>(const DerivDesc*, int, const double*,
                                                   const double*, const double*, const Dims&,
                                                   double*, double*, cudaStream_t);

// Per-block partial sums an edge-derivative launch needs (per branch, twice),
// for the variant with the most blocks.
int deriv_blocks(const Dims& d) {
    if (deriv4_shape(d)) return (d.P + kRB / d.C - 1) / (kRB / d.C);
    return reduction_blocks(d.P);
}

cudaError_t launch_accumulate_scale(double* cum, const double* pool, const int* d_idx, int n,
                                    int Pp, int P, double sign, int log_scalers, int p_begin,
                                    int p_end, cudaStream_t s) {
    (void)P;
    if (n == 0 || p_end <= p_begin) return cudaSuccess;
    const int cnt = p_end - p_begin;
    k_accumulate_scale<<<(cnt + 255) / 256, 256, 0, s>>>(cum, pool, d_idx, n, Pp, p_begin, p_end,
                                                         sign, log_scalers);
    return cudaGetLastError();
}

int deriv4_batch_tile(int C) { return kRB / C * 2; }

template <typename Real>
cudaError_t launch_deriv4_batch(const DerivSeg* d_segs, int nseg, int ncta, int C,
                                cudaStream_t s) {
    if (nseg == 0 || ncta == 0) return cudaSuccess;
    switch (C) {
        case 1: k_deriv4_batch<Real, 1><<<ncta, kRB, 0, s>>>(d_segs, nseg); break;
        case 2: k_deriv4_batch<Real, 2><<<ncta, kRB, 0, s>>>(d_segs, nseg); break;
        case 4: k_deriv4_batch<Real, 4><<<ncta, kRB, 0, s>>>(d_segs, nseg); break;
        case 8: k_deriv4_batch<Real, 8><<<ncta, kRB, 0, s>>>(d_segs, nseg); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_root_batch(const RootSeg* d_segs, int nseg, int ncta, cudaStream_t s) {
    if (nseg == 0 || ncta == 0) return cudaSuccess;
    k_root_batch<Real><<<ncta, kRB, 0, s>>>(d_segs, nseg);
    return cudaGetLastError();
}

int accumulate_batch_patterns() { return 256; }

cudaError_t launch_accumulate_batch(const AccSeg* d_segs, int nseg, int ncta, cudaStream_t s) {
    if (nseg == 0 || ncta == 0) return cudaSuccess;
    k_accumulate_batch<<<ncta, 256, 0, s>>>(d_segs, nseg);
    return cudaGetLastError();
}

cudaError_t launch_final_batch(const FinalSeg* d_segs, int nseg, int nout, cudaStream_t s) {
    if (nseg == 0 || nout == 0) return cudaSuccess;
    k_final_batch<<<nout, kRB, 0, s>>>(d_segs, nseg);
    return cudaGetLastError();
}

template cudaError_t launch_deriv4_batch<float>(const DerivSeg*, int, int, int, cudaStream_t);
template cudaError_t launch_deriv4_batch<double>(const DerivSeg*, int, int, int, cudaStream_t);
template cudaError_t launch_root_batch<float>(const RootSeg*, int, int, cudaStream_t);
template cudaError_t launch_root_batch<double>(const RootSeg*, int, int, cudaStream_t);

#define INST(R)                                                                                  \
    template cudaError_t launch_root_lnl<R>(const void*, const double*, const double*,           \
                                            const double*, const double*, const Dims&, double*,  \
                                            double*, double*, cudaStream_t, bool);               \
    template cudaError_t launch_root_lnl_range<R>(const void*, const double*, const double*,     \
                                                  const double*, const double*, const Dims&,     \
                                                  int, int, double*, double*, double*,           \
                                                  cudaStream_t, bool);                           \
    template cudaError_t launch_edge_lnl<R>(const void*, const void*, int, const void*, double,  \
                                            const void*, double, const void*, double,            \
                                            const double*, const double*, const double*,         \
                                            const double*, const Dims&, double*, double*,        \
                                            double*, double*, double*, cudaStream_t);            \
    template cudaError_t launch_edge_lnl_range<R>(                                               \
        const void*, const void*, int, const void*, double, const void*, double, const void*,    \
        double, const double*, const double*, const double*, const double*, const Dims&, int,    \
        int, double*, double*, double*, double*, double*, cudaStream_t);                         \
    template cudaError_t launch_edge_derivatives<R>(const DerivDesc*, int, const double*,        \
                                                    const double*, const Dims&, double*,         \
                                                    double*, double*, cudaStream_t, int);
INST(float)
INST(double)
#undef INST

}  // namespace b200
