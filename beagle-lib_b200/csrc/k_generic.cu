// Partials and edge derivatives for a general state count (S <= 64), on CUDA
// cores: the FP64 path for every S != 4, and the mixed path's fallback.
//
// Work decomposition.  A thread-block cluster owns one pattern tile; CTA r of
// the cluster owns rate category r (cluster size = C <= 8).  Every CTA walks
// the whole op list for its (tile, category), so dependent ops need no
// grid-wide synchronisation, and the C-fold split keeps enough CTAs in flight
// at the modest pattern counts of 20- and 61-state data.  The per-pattern
// rescaling maximum over categories (CPU/BeagleCPUImpl.hpp:4008-4056) is
// exchanged between the cluster's CTAs through distributed shared memory, so
// each CTA scales its outputs in registers and stores them once.
//
// Per op, one CTA computes a TP x Sg output tile of one category as register
// tiles: each thread owns 4 patterns x 4 states and accumulates
//   y[p][i] = sum_k X[p][k] * A[k][i]
// from shared memory, X being the child's tile in its natural [pattern][state]
// layout and A = P^T (so A's rows are contiguous).  Both are staged with
// cp.async into a two-stage buffer; the next op's operands are prefetched
// during the current op whenever the next op does not read this op's output.
// Matrices come from their transposed device images (k_matrices.cu keeps
// P and P^T), so no shared-memory transposes are needed.
#include <cooperative_groups.h>

#include "b200_kernels.h"
#include "b200_vec.cuh"

namespace cg = cooperative_groups;

namespace b200 {
namespace {

template <typename Real, int SPAD>
struct GCfg {
    // Patterns per tile: the largest that keeps two operand stages in shared
    // memory and at most 256 threads.
    static constexpr int TP = (sizeof(Real) == 4) ? (SPAD >= 48 ? 64 : 128)
                                                  : (SPAD >= 64 ? 32 : SPAD >= 48 ? 64 : 128);
    static constexpr int SG = SPAD / 4;            // state groups (4 states each)
    static constexpr int PG = TP / 4;              // pattern groups (4 patterns each)
    static constexpr int NT = SG * PG;             // threads per CTA
    static constexpr int XS = SPAD + 4;            // padded tile row (elements)
    static constexpr int MAT = SPAD * SPAD;
    static constexpr int TILE = TP * XS;
    static constexpr int STAGE = 2 * MAT + 2 * TILE;
    static constexpr int CH = 16 / sizeof(Real);   // elements per 16-byte chunk
    static size_t smem() { return sizeof(Real) * (2 * STAGE + TP * SG + 2 * TP); }
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = pred ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_one() {
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// A[SPAD][SPAD] <- M[Sg][Sg] (row-major image), zero beyond Sg.
template <typename Real, int SPAD>
__device__ __forceinline__ void stage_mat(Real* A, const Real* M, int Sg, int tid, int nt) {
    using G = GCfg<Real, SPAD>;
    constexpr int CPR = SPAD / G::CH;                       // chunks per row
    for (int q = tid; q < SPAD * CPR; q += nt) {
        const int r = q / CPR, k = (q - r * CPR) * G::CH;
        const bool ok = r < Sg && k < Sg;
        cp_async16(A + r * SPAD + k, ok ? (const void*)(M + r * Sg + k) : (const void*)M, ok);
    }
}

// X[TP][XS] <- rows p0..p0+TP of category c of a partials buffer.
template <typename Real, int SPAD>
__device__ __forceinline__ void stage_tile(Real* X, const Real* src, int p0, int c, int C, int Sg,
                                           int tid, int nt) {
    using G = GCfg<Real, SPAD>;
    constexpr int CPR = SPAD / G::CH;
    for (int q = tid; q < G::TP * CPR; q += nt) {
        const int p = q / CPR, k = (q - p * CPR) * G::CH;
        const bool ok = k < Sg;
        const Real* g = src + ((size_t)(p0 + p) * C + c) * Sg + k;
        cp_async16(X + p * G::XS + k, ok ? (const void*)g : (const void*)src, ok);
    }
}

template <typename Real>
__device__ __forceinline__ void lds4(const Real* p, Real v[4]) {
    if (sizeof(Real) == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
        const double2 a = reinterpret_cast<const double2*>(p)[0];
        const double2 b = reinterpret_cast<const double2*>(p)[1];
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
}

// acc[q][r] = sum_{k < K} X[pl + q][k] * A[k][i0 + r]
template <typename Real, int SPAD>
__device__ __forceinline__ void mm4x4(const Real* X, const Real* A, int K, int pl, int i0,
                                      Real acc[4][4]) {
    using G = GCfg<Real, SPAD>;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r] = 0;
    for (int k = 0; k < K; k += 4) {
        Real x[4][4], a[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q) lds4(X + (pl + q) * G::XS + k, x[q]);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) lds4(A + (k + kk) * SPAD + i0, a[kk]);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int r = 0; r < 4; ++r) acc[q][r] += x[q][kk] * a[kk][r];
    }
}

// Operand from compact tip states: y[q][r] = A[s_q][i0 + r] (= P[i][s]), pad if missing.
template <typename Real, int SPAD>
__device__ __forceinline__ void tip4x4(const Real* A, const int s[4], int S, Real pad, int i0,
                                       Real acc[4][4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        Real a[4];
        lds4(A + (s[q] < S ? s[q] : 0) * SPAD + i0, a);
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r] = (s[q] < S) ? a[r] : pad;
    }
}

// Per-pattern maximum over the cluster's categories of out[q][r] (states < S).
// Threads of one pattern group reduce through `red`, CTAs through DSMEM.
// `smax` alternates between two buffers (the caller passes rescaling k's
// buffer k & 1), so one cluster barrier per rescaling suffices: a CTA writes
// a buffer again only after the next rescaling's barrier, which every CTA of
// the cluster reaches after its reads of that buffer.  The walk ends with a
// cluster barrier, so no CTA exits while another reads its buffer.
template <typename Real, int SPAD>
__device__ __forceinline__ void cluster_max(const Real out[4][4], int S, int i0, int pg, int sg,
                                            Real* red, Real* smax, int C, Real m[4]) {
    using G = GCfg<Real, SPAD>;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        Real v = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (i0 + r < S) v = out[q][r] > v ? out[q][r] : v;
        red[(pg * 4 + q) * G::SG + sg] = v;
    }
    __syncthreads();
    if (sg == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            Real v = 0;
            for (int g = 0; g < G::SG; ++g) {
                const Real u = red[(pg * 4 + q) * G::SG + g];
                v = u > v ? u : v;
            }
            smax[pg * 4 + q] = v;
        }
    }
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        Real v = 0;
        for (int r = 0; r < C; ++r) {
            const Real* rem = cluster.map_shared_rank(smax, r);
            const Real u = rem[pg * 4 + q];
            v = u > v ? u : v;
        }
        m[q] = v;
    }
}

// Shared epilogue of post- and pre-order ops: optional rescale (cluster-wide
// maximum), optional fixed scaling, store of the thread's 4 x 4 tile.
template <typename Real, int SPAD>
__device__ __forceinline__ void finish_tile(const OpDesc& op, Real out[4][4], int p0, int pl,
                                            int i0, int pg, int sg, int c, int S, int Sg, int C,
                                            Real* s_red, Real* s_max, double* cum,
                                            int log_scalers) {
    if (op.cum) cum = op.cum;
    if (op.scale_write) {
        Real m[4];
        cluster_max<Real, SPAD>(out, S, i0, pg, sg, s_red, s_max, C, m);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            Real mq = m[q] == Real(0) ? Real(1) : m[q];
            const Real inv = recip(mq);
#pragma unroll
            for (int r = 0; r < 4; ++r) out[q][r] *= inv;
            const int p = p0 + pl + q;
            if (c == 0 && sg == 0 && p >= op.p_begin && p < op.p_end) {
                const double lm = scale_log(mq);
                op.scale_write[p] = log_scalers ? lm : (double)mq;
                if (cum) cum[p] += lm;
            }
        }
    } else if (op.scale_read) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const Real inv = recip((Real)op.scale_read[p0 + pl + q]);
#pragma unroll
            for (int r = 0; r < 4; ++r) out[q][r] *= inv;
        }
    }
    if (i0 < Sg) {
        Real* d = static_cast<Real*>(op.dest);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int p = p0 + pl + q;
            if (p >= op.p_begin && p < op.p_end)
                st4(d + ((size_t)p * C + c) * Sg + i0, out[q]);
        }
    }
}

// Issue the cp.async loads of one op's operands into stage `st`.
//   post: A1 = P1^T, A2 = P2^T, X1, X2 (partials children only)
//   pre:  A2 = P_sib^T, X2 = sibling (partials only), A1 = P_node (natural)
template <typename Real, int SPAD, bool PRE>
__device__ __forceinline__ void issue_op(const OpDesc& op, Real* stage, int p0, int c, int C,
                                         int Sg, int tid, int nt) {
    using G = GCfg<Real, SPAD>;
    Real* A1 = stage;
    Real* A2 = stage + G::MAT;
    Real* X1 = stage + 2 * G::MAT;
    Real* X2 = X1 + G::TILE;
    const size_t mo = (size_t)c * Sg * Sg;
    if (PRE) {
        const Real* mnat = static_cast<const Real*>(
            (op.kind & kM1Transposed) ? op.m1t : op.m1);   // want P[i][j]
        stage_mat<Real, SPAD>(A1, mnat + mo, Sg, tid, nt);
    } else {
        stage_mat<Real, SPAD>(A1, static_cast<const Real*>(op.m1t) + mo, Sg, tid, nt);
        if (!(op.kind & kX1States))
            stage_tile<Real, SPAD>(X1, static_cast<const Real*>(op.x1), p0, c, C, Sg, tid, nt);
    }
    stage_mat<Real, SPAD>(A2, static_cast<const Real*>(op.m2t) + mo, Sg, tid, nt);
    if (!(op.kind & kX2States))
        stage_tile<Real, SPAD>(X2, static_cast<const Real*>(op.x2), p0, c, C, Sg, tid, nt);
    cp_async_commit();
}

template <typename Real, int SPAD, bool PRE>
__global__ void __launch_bounds__(GCfg<Real, SPAD>::NT)
k_opwalk_x(const OpDesc* __restrict__ ops, const uint8_t* __restrict__ dep_prev, int nops, int S,
           int Sg, int C, double* cum, int log_scalers) {
    using G = GCfg<Real, SPAD>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real* stages = reinterpret_cast<Real*>(smem_raw);
    Real* s_red = stages + 2 * G::STAGE;     // [TP][SG]
    Real* s_max = s_red + G::TP * G::SG;     // [2][TP], alternating per rescaling
    const int tid = threadIdx.x;
    const int sg = tid % G::SG, pg = tid / G::SG;
    const int i0 = sg * 4, pl = pg * 4;
    const int c = blockIdx.x % C;
    const int p0 = (blockIdx.x / C) * G::TP;
    if (nops == 0) return;
    issue_op<Real, SPAD, PRE>(ops[0], stages, p0, c, C, Sg, tid, G::NT);
    int cur = 0;
    int nresc = 0;   // rescalings so far: rescaling k uses s_max buffer k & 1
    for (int o = 0; o < nops; ++o) {
        const OpDesc op = ops[o];
        const bool next = o + 1 < nops;
        const bool early = next && !dep_prev[o + 1];
        if (early) {
            issue_op<Real, SPAD, PRE>(ops[o + 1], stages + (cur ^ 1) * G::STAGE, p0, c, C, Sg, tid,
                                      G::NT);
            cp_async_wait_one();
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        Real* st = stages + cur * G::STAGE;
        const Real* A1 = st;
        const Real* A2 = st + G::MAT;
        const Real* X1 = st + 2 * G::MAT;
        Real* X2 = st + 2 * G::MAT + G::TILE;
        Real out[4][4];
        int s2[4];
        if (op.kind & kX2States) {
#pragma unroll
            for (int q = 0; q < 4; ++q) s2[q] = static_cast<const int*>(op.x2)[p0 + pl + q];
        }
        if (!PRE) {
            Real y2[4][4];
            if (op.kind & kX1States) {
                int s1[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) s1[q] = static_cast<const int*>(op.x1)[p0 + pl + q];
                tip4x4<Real, SPAD>(A1, s1, S, (Real)op.pad1, i0, out);
            } else {
                mm4x4<Real, SPAD>(X1, A1, Sg, pl, i0, out);
            }
            if (op.kind & kX2States) tip4x4<Real, SPAD>(A2, s2, S, (Real)op.pad2, i0, y2);
            else mm4x4<Real, SPAD>(X2, A2, Sg, pl, i0, y2);
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int r = 0; r < 4; ++r) out[q][r] *= y2[q][r];
        } else {
            // z = pre_parent (.) (P_sib . x_sib), written over the sibling tile
            Real z[4][4];
            if (op.kind & kX2States) tip4x4<Real, SPAD>(A2, s2, S, (Real)op.pad2, i0, z);
            else mm4x4<Real, SPAD>(X2, A2, Sg, pl, i0, z);
            const Real* par = static_cast<const Real*>(op.x1);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                Real pv[4] = {0, 0, 0, 0};
                if (i0 < Sg) ld4(par + ((size_t)(p0 + pl + q) * C + c) * Sg + i0, pv);
#pragma unroll
                for (int r = 0; r < 4; ++r) z[q][r] *= pv[r];
            }
            __syncthreads();   // every thread is done reading X2
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int r = 0; r < 4; ++r) X2[(pl + q) * G::XS + i0 + r] = z[q][r];
            __syncthreads();
            // dest[p][j] = sum_i z[p][i] P[i][j]
            mm4x4<Real, SPAD>(X2, A1, Sg, pl, i0, out);
        }
        finish_tile<Real, SPAD>(op, out, p0, pl, i0, pg, sg, c, S, Sg, C, s_red,
                                s_max + (nresc & 1) * G::TP, PRE ? nullptr : cum, log_scalers);
        if (op.scale_write) ++nresc;
        __syncthreads();   // stage `cur` free, stores of this op visible to the CTA
        if (next && !early)
            issue_op<Real, SPAD, PRE>(ops[o + 1], stages + (cur ^ 1) * G::STAGE, p0, c, C, Sg, tid,
                                      G::NT);
        cur ^= 1;
    }
    // no CTA leaves while another reads its s_max through DSMEM
    cg::this_cluster().sync();
}

// Edge derivatives: cluster = (pattern tile, branch), CTA = category.
// num_c[p] = sum_k pre[p][k] (D_c . post)[p][k], den_c[p] = sum_k pre[p][k] post[p][k],
// combined over categories with the category weights in FP64 through DSMEM.
template <typename Real, int SPAD>
__global__ void __launch_bounds__(GCfg<Real, SPAD>::NT)
k_deriv_x(const DerivDesc* __restrict__ desc, const double* __restrict__ catw,
          const double* __restrict__ patw, int S, int Sg, int C, int P, int ntiles, double* site,
          double* block) {
    using G = GCfg<Real, SPAD>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real* A = reinterpret_cast<Real*>(smem_raw);
    Real* X = A + G::MAT;
    double* s_nd = reinterpret_cast<double*>(X + G::TILE);    // [TP][SG][2]
    double* s_tot = s_nd + 2 * G::TP * G::SG;                 // [TP][2] per CTA
    const int tid = threadIdx.x;
    const int sg = tid % G::SG, pg = tid / G::SG;
    const int i0 = sg * 4, pl = pg * 4;
    const int c = blockIdx.x % C;
    const int tile = (blockIdx.x / C) % ntiles;
    const int b = blockIdx.x / (C * ntiles);
    const int p0 = tile * G::TP;
    const DerivDesc dd = desc[b];
    const size_t mo = (size_t)c * Sg * Sg;
    stage_mat<Real, SPAD>(A, static_cast<const Real*>(dd.dmatt) + mo, Sg, tid, G::NT);
    if (!dd.post_is_states)
        stage_tile<Real, SPAD>(X, static_cast<const Real*>(dd.post), p0, c, C, Sg, tid, G::NT);
    cp_async_commit();
    Real pre[4][4];
    const Real* pr = static_cast<const Real*>(dd.pre);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        pre[q][0] = pre[q][1] = pre[q][2] = pre[q][3] = 0;
        if (i0 < Sg) ld4(pr + ((size_t)(p0 + pl + q) * C + c) * Sg + i0, pre[q]);
    }
    int s[4] = {0, 0, 0, 0};
    if (dd.post_is_states) {
#pragma unroll
        for (int q = 0; q < 4; ++q) s[q] = static_cast<const int*>(dd.post)[p0 + pl + q];
    }
    cp_async_wait_all();
    __syncthreads();
    Real y[4][4];
    if (dd.post_is_states) tip4x4<Real, SPAD>(A, s, S, (Real)dd.dpad, i0, y);
    else mm4x4<Real, SPAD>(X, A, Sg, pl, i0, y);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        Real n = 0, d = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int i = i0 + r;
            if (i >= S) continue;
            Real xv;
            if (dd.post_is_states) xv = (s[q] >= S || s[q] == i) ? Real(1) : Real(0);
            else xv = X[(pl + q) * G::XS + i];
            n += pre[q][r] * y[q][r];
            d += pre[q][r] * xv;
        }
        s_nd[((pl + q) * G::SG + sg) * 2 + 0] = (double)n;
        s_nd[((pl + q) * G::SG + sg) * 2 + 1] = (double)d;
    }
    __syncthreads();
    const double w = catw[c];
    if (sg == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double n = 0, d = 0;
            for (int g = 0; g < G::SG; ++g) {
                n += s_nd[((pl + q) * G::SG + g) * 2 + 0];
                d += s_nd[((pl + q) * G::SG + g) * 2 + 1];
            }
            s_tot[(pl + q) * 2 + 0] = w * n;
            s_tot[(pl + q) * 2 + 1] = w * d;
        }
    }
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    if (c == 0) {
        // rank 0: combine categories, per-site value, weighted sums for the tile
        double v1 = 0, v2 = 0;
        for (int pl2 = tid; pl2 < G::TP; pl2 += G::NT) {
            double n = 0, d = 0;
            for (int r = 0; r < C; ++r) {
                const double* rem = cluster.map_shared_rank(s_tot, r);
                n += rem[pl2 * 2 + 0];
                d += rem[pl2 * 2 + 1];
            }
            const int p = p0 + pl2;
            if (p < P) {
                const double dv = n / d;
                if (site) site[(size_t)b * P + p] = dv;
                v1 += dv * patw[p];
                v2 += dv * dv * patw[p];
            }
        }
        // block reduction (fixed order) of v1, v2 over the CTA's threads: the
        // 32 threads of warp 0 each add a strided subset, then a shuffle tree
        // (NT need not be a multiple of 32)
        double* red = s_nd;   // reuse: [NT][2]
        red[tid * 2 + 0] = v1;
        red[tid * 2 + 1] = v2;
        __syncthreads();
        if (tid < 32) {
            double t1 = 0, t2 = 0;
            for (int k = tid; k < G::NT; k += 32) {
                t1 += red[k * 2 + 0];
                t2 += red[k * 2 + 1];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                t1 += __shfl_xor_sync(0xffffffffu, t1, o);
                t2 += __shfl_xor_sync(0xffffffffu, t2, o);
            }
            if (tid == 0) {
                const int nb = gridDim.x / (C * ntiles);
                block[(size_t)b * ntiles + tile] = t1;
                block[(size_t)(nb + b) * ntiles + tile] = t2;
            }
        }
    }
    cluster.sync();   // remote reads done before any CTA of the cluster exits
}

template <typename K, typename... Args>
cudaError_t launch_clustered(K kernel, int grid, int threads, size_t smem, int cluster,
                             cudaStream_t s, Args... args) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename Real, int SPAD, bool PRE>
cudaError_t run_opwalk(const OpDesc* ops, const uint8_t* dep, int nops, const Dims& d,
                       double* cum, int ls, cudaStream_t s) {
    using G = GCfg<Real, SPAD>;
    const int ntiles = d.Pp / G::TP;
    return launch_clustered(k_opwalk_x<Real, SPAD, PRE>, ntiles * d.C, G::NT, G::smem(), d.C, s,
                            ops, dep, nops, d.S, d.Sg, d.C, cum, ls);
}

template <typename Real, int SPAD>
cudaError_t run_deriv(const DerivDesc* desc, int nb, const double* catw, const double* patw,
                      const Dims& d, double* site, double* block, cudaStream_t s) {
    using G = GCfg<Real, SPAD>;
    const int ntiles = d.Pp / G::TP;
    const size_t smem = sizeof(Real) * (G::MAT + G::TILE) +
                        sizeof(double) * (2 * G::TP * G::SG + 2 * G::TP + 2 * G::NT);
    return launch_clustered(k_deriv_x<Real, SPAD>, ntiles * d.C * nb, G::NT, smem, d.C, s, desc,
                            catw, patw, d.S, d.Sg, d.C, d.P, ntiles, site, block);
}

}  // namespace

#define B200_SPAD_DISPATCH(Sg, CALL)          \
    ((Sg) <= 8    ? CALL(8)                   \
     : (Sg) <= 16 ? CALL(16)                  \
     : (Sg) <= 24 ? CALL(24)                  \
     : (Sg) <= 32 ? CALL(32)                  \
     : (Sg) <= 48 ? CALL(48)                  \
     : (Sg) <= 64 ? CALL(64)                  \
                  : cudaErrorInvalidValue)

template <typename Real>
cudaError_t launch_opwalk_generic(const OpDesc* ops, const uint8_t* dep, int nops, bool pre,
                                  const Dims& d, double* cum, int ls, cudaStream_t s) {
    if (nops == 0) return cudaSuccess;
    if (d.C > 8) return cudaErrorInvalidValue;
#define POST_(SP) run_opwalk<Real, SP, false>(ops, dep, nops, d, cum, ls, s)
#define PRE_(SP) run_opwalk<Real, SP, true>(ops, dep, nops, d, nullptr, ls, s)
    return pre ? B200_SPAD_DISPATCH(d.Sg, PRE_) : B200_SPAD_DISPATCH(d.Sg, POST_);
#undef POST_
#undef PRE_
}

template <typename Real>
cudaError_t launch_deriv_generic(const DerivDesc* desc, int nb, const double* catw,
                                 const double* patw, const Dims& d, double* site, double* block,
                                 cudaStream_t s) {
    if (nb == 0) return cudaSuccess;
    if (d.C > 8) return cudaErrorInvalidValue;
#define DER_(SP) run_deriv<Real, SP>(desc, nb, catw, patw, d, site, block, s)
    return B200_SPAD_DISPATCH(d.Sg, DER_);
#undef DER_
}

int generic_tile_patterns(int Sg, bool dbl) {
    auto tp = [&](int spad) {
        return dbl ? (spad >= 64 ? 32 : spad >= 48 ? 64 : 128) : (spad >= 48 ? 64 : 128);
    };
    const int spad = Sg <= 8 ? 8 : Sg <= 16 ? 16 : Sg <= 24 ? 24 : Sg <= 32 ? 32 : Sg <= 48 ? 48 : 64;
    return tp(spad);
}

template cudaError_t launch_opwalk_generic<float>(const OpDesc*, const uint8_t*, int, bool,
                                                  const Dims&, double*, int, cudaStream_t);
template cudaError_t launch_opwalk_generic<double>(const OpDesc*, const uint8_t*, int, bool,
                                                   const Dims&, double*, int, cudaStream_t);
template cudaError_t launch_deriv_generic<float>(const DerivDesc*, int, const double*,
                                                 const double*, const Dims&, double*, double*,
                                                 cudaStream_t);
template cudaError_t launch_deriv_generic<double>(const DerivDesc*, int, const double*,
                                                  const double*, const Dims&, double*, double*,
                                                  cudaStream_t);

}  // namespace b200
