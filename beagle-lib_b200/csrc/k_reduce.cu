// Pattern reductions: root and edge log-likelihoods, edge derivatives and
// scale-factor accumulation.  All sums that leave the device are FP64 and
// deterministic: fixed 128-thread blocks reduce by warp shuffles and shared
// memory into per-block partial sums, and a second pass (one CTA per output)
// adds the partials in a fixed order.
#include "b200_kernels.h"
#include "b200_vec.cuh"

namespace b200 {

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

template <typename Real>
__global__ void __launch_bounds__(kRB)
k_root_lnl(const Real* __restrict__ root, const double* __restrict__ catw,
           const double* __restrict__ freqs, const double* __restrict__ cum,
           const double* __restrict__ patw, int S, int Sg, int C, int p_begin, int p_end,
           double* site, double* block) {
    __shared__ double sh[kRB / 32];
    const int p = p_begin + blockIdx.x * kRB + threadIdx.x;
    double v = 0;
    if (p < p_end) {
        double l = log(integrate_site(root, catw, freqs, S, Sg, C, p));
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
           int C, int P, double* site, double* site1, double* site2, double* block) {
    __shared__ double sh[kRB / 32];
    const int p = blockIdx.x * kRB + threadIdx.x;
    double v0 = 0, v1 = 0, v2 = 0;
    if (p < P) {
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
// pattern combine their weighted terms with shuffles.  Each thread covers PPT
// patterns kRB / C apart, so a CTA covers kRB / C * PPT patterns and pays its
// two block reductions once for all of them; blockIdx.y = branch.  The
// category's 4x4 derivative matrix is held in registers across the PPT
// patterns.
template <typename Real, int C, int PPT>
__global__ void __launch_bounds__(kRB)
k_edge_deriv4(const DerivDesc* __restrict__ desc, const double* __restrict__ catw,
              const double* __restrict__ patw, int P, double* site, double* block) {
    __shared__ double sh[kRB / 32];
    constexpr int kSlots = kRB / C;
    const int b = blockIdx.y;
    const int c = threadIdx.x % C;
    const int p0 = blockIdx.x * (kSlots * PPT) + threadIdx.x / C;
    const DerivDesc& dd = desc[b];
    const Real* D = static_cast<const Real*>(dd.dmat) + c * 16;
    Real dm[16];
#pragma unroll
    for (int k = 0; k < 4; ++k) ld4(D + 4 * k, dm + 4 * k);
    const double w = catw[c];
    Real z[PPT][4], x[PPT][4];
    int st[PPT];
    const bool states = dd.post_is_states;
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        const int pc = min(p0 + j * kSlots, P - 1);
        ld4(static_cast<const Real*>(dd.pre) + ((size_t)pc * C + c) * 4, z[j]);
        if (states)
            st[j] = static_cast<const int*>(dd.post)[pc];
        else
            ld4(static_cast<const Real*>(dd.post) + ((size_t)pc * C + c) * 4, x[j]);
    }
    double s1 = 0, s2 = 0;
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        const int p = p0 + j * kSlots;
        Real n = 0, q = 0;
        if (states) {
            const int s = st[j];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                Real dk = (Real)dd.dpad;
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (s == i) dk = dm[k * 4 + i];
                n += z[j][k] * dk;
                q += (s >= 4 || k == s) ? z[j][k] : Real(0);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const Real y = dm[k * 4] * x[j][0] + dm[k * 4 + 1] * x[j][1] +
                               dm[k * 4 + 2] * x[j][2] + dm[k * 4 + 3] * x[j][3];
                n += z[j][k] * y;
                q += z[j][k] * x[j][k];
            }
        }
        double num = w * (double)n, den = w * (double)q;
#pragma unroll
        for (int o = 1; o < C; o <<= 1) {
            num += __shfl_xor_sync(0xffffffffu, num, o);
            den += __shfl_xor_sync(0xffffffffu, den, o);
        }
        if (c == 0 && p < P) {
            const double d = num / den;
            if (site) site[(size_t)b * P + p] = d;
            const double wp = patw[p];
            s1 += d * wp;
            s2 += d * d * wp;
        }
    }
    const int nblk = gridDim.x;
    double t = block_sum(s1, sh);
    if (threadIdx.x == 0) block[(size_t)b * nblk + blockIdx.x] = t;
    t = block_sum(s2, sh);
    if (threadIdx.x == 0) block[(size_t)(gridDim.y + b) * nblk + blockIdx.x] = t;
}

__global__ void k_accumulate_scale(double* cum, const double* __restrict__ pool,
                                   const int* __restrict__ idx, int n, int Pp, int p_begin,
                                   int p_end, double sign, int log_scalers) {
    const int p = p_begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= p_end) return;
    double acc = 0;
    for (int i = 0; i < n; ++i) {
        const double v = pool[(size_t)idx[i] * Pp + p];
        acc += log_scalers ? v : log(v);
    }
    cum[p] += sign * acc;
}

}  // namespace

int reduction_blocks(int Pp) { return (Pp + kRB - 1) / kRB; }

template <typename Real>
cudaError_t launch_root_lnl(const void* root, const double* catw, const double* freqs,
                            const double* cum, const double* patw, const Dims& d,
                            double* d_site, double* d_block, double* d_out, cudaStream_t s) {
    return launch_root_lnl_range<Real>(root, catw, freqs, cum, patw, d, 0, d.P, d_site, d_block,
                                       d_out, s);
}

template <typename Real>
cudaError_t launch_root_lnl_range(const void* root, const double* catw, const double* freqs,
                                  const double* cum, const double* patw, const Dims& d,
                                  int p_begin, int p_end, double* d_site, double* d_block,
                                  double* d_out, cudaStream_t s) {
    const int nblk = reduction_blocks(p_end - p_begin);
    if (nblk == 0) return cudaMemsetAsync(d_out, 0, sizeof(double), s);
    k_root_lnl<Real><<<nblk, kRB, 0, s>>>(static_cast<const Real*>(root), catw, freqs, cum, patw,
                                          d.S, d.Sg, d.C, p_begin, p_end, d_site, d_block);
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
    const int nblk = reduction_blocks(d.P);
    k_edge_lnl<Real><<<nblk, kRB, 0, s>>>(
        static_cast<const Real*>(parent), child, child_is_states, static_cast<const Real*>(pmat),
        ppad, static_cast<const Real*>(d1mat), d1pad, static_cast<const Real*>(d2mat), d2pad,
        catw, freqs, cum, patw, d.S, d.Sg, d.C, d.P, d_site, d_site1, d_site2, d_block);
    k_final_sum<<<3, kRB, 0, s>>>(d_block, nblk, 3, d_out);
    return cudaGetLastError();
}

namespace {

bool deriv4_shape(const Dims& d) {
    return d.S == 4 && d.Sg == 4 && (d.C == 1 || d.C == 2 || d.C == 4 || d.C == 8);
}

// Patterns per thread of variant v of the S = 4 derivative kernel.
int deriv4_ppt(int v) { return v <= 0 ? 1 : v == 1 ? 2 : v == 2 ? 4 : 8; }

template <typename Real, int C>
void run_deriv4(int ppt, dim3 grid, cudaStream_t s, const DerivDesc* desc, const double* catw,
                const double* patw, int P, double* site, double* block) {
    switch (ppt) {
        case 1: k_edge_deriv4<Real, C, 1><<<grid, kRB, 0, s>>>(desc, catw, patw, P, site, block); break;
        case 2: k_edge_deriv4<Real, C, 2><<<grid, kRB, 0, s>>>(desc, catw, patw, P, site, block); break;
        case 4: k_edge_deriv4<Real, C, 4><<<grid, kRB, 0, s>>>(desc, catw, patw, P, site, block); break;
        default: k_edge_deriv4<Real, C, 8><<<grid, kRB, 0, s>>>(desc, catw, patw, P, site, block); break;
    }
}

}  // namespace

int deriv4_variants(const Dims& d) { return deriv4_shape(d) ? 4 : 1; }

template <typename Real>
cudaError_t launch_edge_derivatives(const DerivDesc* desc, int nb, const double* catw,
                                    const double* patw, const Dims& d, double* d_site,
                                    double* d_block, double* d_sums, cudaStream_t s,
                                    int variant) {
    if (nb == 0) return cudaSuccess;
    int nblk = reduction_blocks(d.P);
    if (deriv4_shape(d)) {
        if (variant < 0) variant = d.P >= 32768 ? 2 : 0;
        const int ppt = deriv4_ppt(variant);
        const int ppb = kRB / d.C * ppt;
        nblk = (d.P + ppb - 1) / ppb;
        dim3 grid(nblk, nb);
        switch (d.C) {
            case 1: run_deriv4<Real, 1>(ppt, grid, s, desc, catw, patw, d.P, d_site, d_block); break;
            case 2: run_deriv4<Real, 2>(ppt, grid, s, desc, catw, patw, d.P, d_site, d_block); break;
            case 4: run_deriv4<Real, 4>(ppt, grid, s, desc, catw, patw, d.P, d_site, d_block); break;
            default: run_deriv4<Real, 8>(ppt, grid, s, desc, catw, patw, d.P, d_site, d_block); break;
        }
    } else {
        dim3 grid(nblk, nb);
        k_edge_deriv<Real><<<grid, kRB, 0, s>>>(desc, catw, patw, d.S, d.Sg, d.C, d.P, d_site,
                                                d_block);
    }
    k_final_sum<<<2 * nb, kRB, 0, s>>>(d_block, nblk, 2 * nb, d_sums);
    return cudaGetLastError();
}

cudaError_t launch_deriv_final(const double* d_block, int nblk, int nb, double* d_sums,
                               cudaStream_t s) {
    k_final_sum<<<2 * nb, kRB, 0, s>>>(d_block, nblk, 2 * nb, d_sums);
    return cudaGetLastError();
}

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

#define INST(R)                                                                                  \
    template cudaError_t launch_root_lnl<R>(const void*, const double*, const double*,           \
                                            const double*, const double*, const Dims&, double*,  \
                                            double*, double*, cudaStream_t);                     \
    template cudaError_t launch_root_lnl_range<R>(const void*, const double*, const double*,     \
                                                  const double*, const double*, const Dims&,     \
                                                  int, int, double*, double*, double*,           \
                                                  cudaStream_t);                                 \
    template cudaError_t launch_edge_lnl<R>(const void*, const void*, int, const void*, double,  \
                                            const void*, double, const void*, double,            \
                                            const double*, const double*, const double*,         \
                                            const double*, const Dims&, double*, double*,        \
                                            double*, double*, double*, cudaStream_t);            \
    template cudaError_t launch_edge_derivatives<R>(const DerivDesc*, int, const double*,        \
                                                    const double*, const Dims&, double*,         \
                                                    double*, double*, cudaStream_t, int);
INST(float)
INST(double)
#undef INST

}  // namespace b200
