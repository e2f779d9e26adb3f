// Partials and edge derivatives of the mixed-precision (FP32) path for
// 4 < S <= 64 on the fifth-generation tensor cores (tcgen05, kind::tf32).
//
// Every post-order child, the pre-order sibling and the derivative are the
// same contraction per rate category c and pattern tile:
//     Y[p][i] = sum_k X[p][k] * M[i][k]        (X: 128 patterns x K states)
// i.e. a 128 x N x K GEMM with A = the partials tile (K-major, one pattern per
// row) and B = the matrix rows (K-major).  The pre-order op chains a second
// one: Z = pre_parent (.) (X_sib . P_sib^T), dest = Z . P_node, with Z written
// back to shared memory from registers.
//
// Precision.  tf32 keeps 10 explicit mantissa bits, so both operands are split
// into hi = x with the low 13 mantissa bits cleared (exactly representable)
// and lo = x - hi (exact in FP32), and each K-step issues three MMAs into the
// same FP32 accumulator: hi*hi + hi*lo + lo*hi.  The dropped lo*lo term and
// the tf32 rounding of lo are below 2^-20 relative, the accuracy class of the
// FP32 CUDA-core kernels (k_generic.cu) this path replaces.
//
// Work decomposition (as in k_generic.cu): a thread-block cluster owns one
// 128-pattern tile, CTA r of the cluster owns rate category r, every CTA
// walks the whole op list for its (tile, category), and the rescaling maximum
// over categories (CPU/BeagleCPUImpl.hpp:4008-4056) is exchanged through
// distributed shared memory.  A CTA has 128 threads: thread t owns pattern row
// t, which is TMEM lane t of every accumulator.
//
// Per contraction, K is processed in chunks of KC (<= 32) states: the CTA's
// threads load the A rows and the B rows of the chunk from global memory,
// split them and store both halves in the canonical no-swizzle K-major layout
// (8-row x 16-byte core matrices, LBO = 128 B between the two 16-byte K halves
// of an MMA step, SBO = KC * 32 B between 8-row groups); thread 0 issues the
// MMAs and commits them to an mbarrier, whose completion frees the chunk's
// shared memory for the next one.  Loads of other CTAs on the SM overlap the
// MMAs (up to 4 CTAs per SM).
//
// TMEM: a CTA allocates 2 N (post / pre) or N (derivative) columns, rounded up
// to a power of two.  Every launch reserves shared memory in proportion to
// its columns (tc_smem), so the CTAs resident on one SM, from any mix of
// these launches, can never ask for more than the 512 columns an SM has, and
// an allocation never waits on another cluster's CTA.
//
// Every wait on an mbarrier is bounded (about a second); on time-out the
// thread sets b200_tc_status, stops waiting for the rest of the launch, keeps
// to the same barrier sequence as its cluster and frees its TMEM at the end.
#include <cooperative_groups.h>

#include "b200_kernels.h"
#include <cuda.h>

#include "b200_vec.cuh"

namespace cg = cooperative_groups;

namespace b200 {

__device__ int b200_tc_status;   // nonzero: a tensor-core kernel gave up waiting

namespace {

constexpr int kTM = 128;                    // patterns per tile = MMA M = TMEM lanes
constexpr int kTT = 128;                    // threads per CTA
constexpr long long kWaitCycles = 2000000000LL;

// ------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`.  After one time-out the thread
// stops waiting (`failed` stays set) and the status flag tells the host.
__device__ __forceinline__ void mbar_wait(uint64_t* bar, uint32_t parity, bool& failed) {
    if (failed) return;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > kWaitCycles) {
            failed = true;
            atomicExch(&b200_tc_status, 1);
            return;
        }
    }
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes -> visible to the tensor core's reads.
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accumulate) {
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(mask0),
        "r"(mask1), "r"(mask2), "r"(mask3)
        : "memory");
}

// Arrive once on `bar` when every MMA this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (the warp's 32
// lanes start at `taddr`); the wait is inside the same asm statement, so the
// registers are complete when it returns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor, no swizzle, K-major (sm100 version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: FP32 accumulator, tf32 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
    hi = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
    lo = x - hi;
}

// ------------------------------------------------------------- geometry
// N (output states) padded to 16, K (input states) padded to 8, or to 16 when
// it is split into two chunks; KC = states per K chunk (<= 32).
template <int NP>
struct TcGeo {
    static constexpr int TCOLS = 2 * NP <= 32 ? 32 : 2 * NP <= 64 ? 64 : 128;   // post / pre
    static constexpr int DCOLS = NP <= 32 ? 32 : 64;                           // derivative
};

// K chunking of a state count: K padded to 8 (one chunk) or, above 32
// states, to 16 and split into two chunks of KC = K / 2 = NP / 2 (the
// (NP, KC) pairs of B200_TC_DISPATCH below).
template <int NP>
__host__ __device__ constexpr int chunks_of() { return NP >= 48 ? 2 : 1; }

// Shared memory of one CTA (floats unless noted):
//   A_hi, A_lo [kTM * 32]   B_hi, B_lo [64 * 32]   smax [2][kTM]
//   nd [kTM * 2] doubles, red [kTT * 2] doubles, mbarrier, TMEM address.
struct TcSmem {
    float a_hi[kTM * 32];
    float a_lo[kTM * 32];
    float b_hi[64 * 32];
    float b_lo[64 * 32];
    float smax[2 * kTM];     // alternating per rescaling (see finish_row)
    double nd[kTM * 2];
    double red[kTT * 2];
    uint64_t bar;
    uint32_t tmem;
};

// A K chunk of a contraction is an NROWS x KC block (128 pattern rows of A,
// NP matrix rows of B) stored as hi / lo halves in the canonical layout.  Lane
// l of warp w handles rows 8 w + (l & 7) + 32 gi (gi = 0 .. NROWS / 32 - 1) and
// sixteen-byte columns 4 h + (l >> 3): a store phase of 8 lanes covers the 8
// rows of one core matrix (conflict-free), a warp reads 8 rows x 64 contiguous
// bytes per load, and all offsets but one base per lane are compile-time.
// A has at most 8 pieces per lane (128 rows, KC <= 32), B at most 4 (NP <= 64).
template <int NROWS, int KC>
struct Pieces {
    static constexpr int NKC = KC / 4;               // sixteen-byte columns
    static constexpr int NH = (NKC + 3) / 4;         // column groups of 4
    static constexpr int NG = (NROWS / 8 + 3) / 4;   // row groups per warp
};

// This lane's pieces of chunk [k0, k0 + KC) of a row-major source (row r at
// src + r * rstride; rows >= nvalid and columns >= Sg are zero), all loads
// issued before any is used.
template <int NROWS, int KC, bool RO>
__device__ __forceinline__ void gather(float v[][4], const float* src, size_t rstride, int nvalid,
                                       int k0, int Sg) {
    using PC = Pieces<NROWS, KC>;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = warp * 8 + (lane & 7), c0 = lane >> 3;
    const float* base = src + (size_t)r0 * rstride + k0 + 4 * c0;
#pragma unroll
    for (int gi = 0; gi < PC::NG; ++gi)
#pragma unroll
        for (int h = 0; h < PC::NH; ++h) {
            float* d = v[gi * PC::NH + h];
            d[0] = d[1] = d[2] = d[3] = 0.f;
            const int r = r0 + 32 * gi, kc = 4 * h + c0;
            if (warp + 4 * gi < NROWS / 8 && kc < PC::NKC && r < nvalid && k0 + 4 * kc < Sg) {
                const float* g = base + (size_t)(32 * gi) * rstride + 16 * h;
                if (RO) ldg4(g, d);
                else ld4(g, d);
            }
        }
}

// Split this lane's pieces and store both halves.
template <int NROWS, int KC>
__device__ __forceinline__ void scatter(const float v[][4], float* hi, float* lo) {
    using PC = Pieces<NROWS, KC>;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = (warp * PC::NKC + (lane >> 3)) * 32 + (lane & 7) * 4;
#pragma unroll
    for (int gi = 0; gi < PC::NG; ++gi)
#pragma unroll
        for (int h = 0; h < PC::NH; ++h) {
            if (warp + 4 * gi >= NROWS / 8 || 4 * h + (lane >> 3) >= PC::NKC) continue;
            const float* v4 = v[gi * PC::NH + h];
            float h4[4], l4[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) split_tf32(v4[q], h4[q], l4[q]);
            const int off = s0 + (4 * gi * PC::NKC + 4 * h) * 32;
            st4(hi + off, h4);
            st4(lo + off, l4);
        }
}

// The 128-byte swizzled K-major layout (what TMA's SWIZZLE_128B writes and
// smem_desc_sw128 describes), used for chunks of 32 states: row r of a tile
// is the 128-byte line at r * 128 bytes, and its 16-byte piece kc sits at
// piece kc ^ (r & 7) of that line; tiles start on 1024-byte boundaries.  Lane
// l of warp w handles rows 4 w + (l >> 3) + 16 i and piece l & 7, so one
// warp load covers 4 whole rows (4 x 128 contiguous bytes) and one warp store
// writes each of those rows' 8 pieces to 8 distinct bank groups of its line.
// 16-byte pieces of chunk q that its MMAs read: whole 8-state K steps up to
// Sg (the rest of the 32-state row is never read, so it is neither loaded
// nor stored).
// NP = 64 (49 to 64 states) keeps whole chunks: trimming its second chunk
// would save little and the run-time counts cost the widest walks registers
// they do not have.
template <int NP>
__device__ __forceinline__ int chunk_pieces(int Sg, int q) {
    if constexpr (NP == 64) return 8;
    int k = Sg - 32 * q;
    k = k < 32 ? k : 32;
    return (k + 7) / 8 * 2;
}

template <int NROWS, bool RO>
__device__ __forceinline__ void gather_sw(float v[][4], const float* src, size_t rstride,
                                          int nvalid, int k0, int Sg, int npieces) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = warp * 4 + (lane >> 3), k = k0 + 4 * (lane & 7);
    const bool piece = (lane & 7) < npieces;
    const float* base = src + (size_t)r0 * rstride + k;
#pragma unroll
    for (int i = 0; i < NROWS / 16; ++i) {
        float* d = v[i];
        d[0] = d[1] = d[2] = d[3] = 0.f;
        if (piece && r0 + 16 * i < nvalid && k < Sg) {
            const float* g = base + (size_t)(16 * i) * rstride;
            if (RO) ldg4(g, d);
            else ld4(g, d);
        }
    }
}

template <int NROWS>
__device__ __forceinline__ void scatter_sw(const float v[][4], float* hi, float* lo,
                                           int npieces) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = warp * 4 + (lane >> 3), kc = lane & 7;
    if (kc >= npieces) return;
    // rows r0 + 16 i share r0 & 7, so every piece lands at the same swizzled column
    const int off0 = r0 * 32 + ((kc ^ (r0 & 7)) * 4);
#pragma unroll
    for (int i = 0; i < NROWS / 16; ++i) {
        float h4[4], l4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) split_tf32(v[i][q], h4[q], l4[q]);
        st4(hi + off0 + i * 16 * 32, h4);
        st4(lo + off0 + i * 16 * 32, l4);
    }
}

// Row t of an A tile (swizzled layout) from registers: z[Q 32 .. Q 32 + 32).
template <int NP, int Q>
__device__ __forceinline__ void store_row_sw128(float* hi, float* lo, const float z[NP]) {
    const int t = threadIdx.x;
#pragma unroll
    for (int kc = 0; kc < 8; ++kc) {
        float h4[4], l4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = Q * 32 + kc * 4 + q;
            split_tf32(k < NP ? z[k < NP ? k : 0] : 0.f, h4[q], l4[q]);
        }
        const int off = t * 32 + ((kc ^ (t & 7)) * 4);
        st4(hi + off, h4);
        st4(lo + off, l4);
    }
}

// Shared-memory descriptor of a K-major tile with 128-byte swizzle (sm100
// layout type 2): rows of 128 bytes, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;                       // leading byte offset (unused here)
    d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Chunk helpers for either layout: KC == 32 uses the swizzled layout.
template <int NROWS, int KC, bool RO, int NP>
__device__ __forceinline__ void gather_any(float v[][4], const float* src, size_t rstride,
                                           int nvalid, int k0, int Sg) {
    if constexpr (KC == 32)
        gather_sw<NROWS, RO>(v, src, rstride, nvalid, k0, Sg, chunk_pieces<NP>(Sg, k0 / 32));
    else gather<NROWS, KC, RO>(v, src, rstride, nvalid, k0, Sg);
}

template <int NROWS, int KC, int NP>
__device__ __forceinline__ void scatter_any(const float v[][4], float* hi, float* lo, int Sg,
                                            int q) {
    if constexpr (KC == 32) scatter_sw<NROWS>(v, hi, lo, chunk_pieces<NP>(Sg, q));
    else scatter<NROWS, KC>(v, hi, lo);
}

// One K chunk in flight: this lane's pieces of A and of B.
struct ChunkRegs {
    float a[8][4];
    float b[4][4];
    int s;              // this thread's tip state (one-hot A rows)
};

// One K chunk of a contraction Y[p][i] = sum_k X[p][k] M[i][k]: A rows from
// partials `x`, or (st, 32-state chunks) one-hot rows of the tile's compact
// tip states, so that Y[p][i] = M[i][state p] comes out of the same MMAs; B
// rows from matrix `m` (row stride Sg), the accumulator at TMEM column `col`,
// chunk index `q`.
struct Job {
    const float* x;
    const float* m;
    const int* st;
    uint32_t col;
    int q;
};

template <int NP, int KC, bool ONEHOT>
__device__ __forceinline__ void gather_job(ChunkRegs& cr, const Job& jb, size_t xs, int Sg) {
    if (ONEHOT && jb.st) cr.s = jb.st[threadIdx.x];
    else gather_any<kTM, KC, false, NP>(cr.a, jb.x, xs, kTM, jb.q * KC, Sg);
    gather_any<NP, KC, true, NP>(cr.b, jb.m, Sg, Sg, jb.q * KC, Sg);
}

// Row t of a one-hot A chunk (swizzled layout, hi half only: the lo half of
// 0 and 1 is 0): 1 at state s when s falls in chunk q, zeros elsewhere; a
// missing state (outside [0, S)) is a zero row, and the epilogue puts the
// matrix's pad value in its place.
__device__ __forceinline__ void onehot_row_sw(float* hi, int s, int q, int S) {
    const int t = threadIdx.x;
    const int k = (s >= 0 && s < S) ? s - 32 * q : -1;
#pragma unroll
    for (int kc = 0; kc < 8; ++kc) {
        float v[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) v[e] = (k == 4 * kc + e) ? 1.f : 0.f;
        st4(hi + t * 32 + ((kc ^ (t & 7)) * 4), v);
    }
}

// Row t of A chunk Q from registers: z[Q KC .. Q KC + KC).  Compile-time
// indices keep z in registers.
template <int NP, int KC, int Q>
__device__ __forceinline__ void store_row(float* hi, float* lo, const float z[NP]) {
    constexpr int NKC = KC / 4;
    const int t = threadIdx.x;
    const int s0 = (t >> 3) * NKC * 32 + (t & 7) * 4;
#pragma unroll
    for (int kc = 0; kc < NKC; ++kc) {
        float h4[4], l4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = Q * KC + kc * 4 + q;
            split_tf32(k < NP ? z[k < NP ? k : 0] : 0.f, h4[q], l4[q]);
        }
        st4(hi + s0 + kc * 32, h4);
        st4(lo + s0 + kc * 32, l4);
    }
}

// Issue the 3 x KC / 8 MMAs of one chunk (thread 0 only); `first` clears the
// accumulator with the first MMA.  Completion arrives on sm.bar.
template <int KC, typename SM>
__device__ __forceinline__ void issue_chunk(SM& sm, uint32_t d_tmem, int N, bool first,
                                            bool onehot = false, int ksteps = 4) {
    const uint32_t idesc = idesc_tf32(kTM, N);
    if constexpr (KC == 32) {
        // swizzled tiles: up to 4 K steps of 8 tf32 (32 bytes) along each
        // 128-byte row (only those that hold states < Sg)
        const uint32_t ah = smem_u32(sm.a_hi), al = smem_u32(sm.a_lo);
        const uint32_t bh = smem_u32(sm.b_hi), bl = smem_u32(sm.b_lo);
        tc_fence_after();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k >= ksteps) break;
            const uint32_t o = (uint32_t)k * 32u;
            const uint64_t dah = smem_desc_sw128(ah + o), dal = smem_desc_sw128(al + o);
            const uint64_t dbh = smem_desc_sw128(bh + o), dbl = smem_desc_sw128(bl + o);
            mma_tf32(d_tmem, dah, dbh, idesc, (first && k == 0) ? 0u : 1u);
            mma_tf32(d_tmem, dah, dbl, idesc, 1u);
            if (!onehot) mma_tf32(d_tmem, dal, dbh, idesc, 1u);   // one-hot rows: lo = 0
        }
        mma_commit(&sm.bar);
        return;
    }
    const uint32_t ah = smem_u32(sm.a_hi), al = smem_u32(sm.a_lo);
    const uint32_t bh = smem_u32(sm.b_hi), bl = smem_u32(sm.b_lo);
    constexpr uint32_t sbo = (uint32_t)KC * 32u;   // bytes between 8-row groups
    tc_fence_after();
#pragma unroll
    for (int s = 0; s < KC / 8; ++s) {
        const uint32_t o = (uint32_t)s * 256u;
        const uint64_t dah = smem_desc(ah + o, 128, sbo), dal = smem_desc(al + o, 128, sbo);
        const uint64_t dbh = smem_desc(bh + o, 128, sbo), dbl = smem_desc(bl + o, 128, sbo);
        mma_tf32(d_tmem, dah, dbh, idesc, (first && s == 0) ? 0u : 1u);
        mma_tf32(d_tmem, dah, dbl, idesc, 1u);
        mma_tf32(d_tmem, dal, dbh, idesc, 1u);
    }
    mma_commit(&sm.bar);
}

// Per-CTA state of the MMA pipeline: phase of sm.bar and whether a commit is
// outstanding (the chunk buffers are busy until it completes).
struct Pipe {
    uint32_t phase = 0;
    bool pending = false;
    bool failed = false;
};

template <typename SM>
__device__ __forceinline__ void pipe_drain(SM& sm, Pipe& pp) {
    if (pp.pending) {
        mbar_wait(&sm.bar, pp.phase, pp.failed);
        pp.phase ^= 1u;
        pp.pending = false;
    }
}

// Run up to 4 chunk jobs through the single chunk buffer: the registers of
// job i + 1 are gathered while the MMAs of job i run.
// ONEHOT: jobs may be one-hot tip jobs (32-state chunks only).
template <int NP, int KC, bool ONEHOT = false, typename SM>
__device__ __forceinline__ void run_jobs(SM& sm, Pipe& pp, uint32_t tmem, const Job (&jobs)[4],
                                         int n, size_t xs, int Sg, int S, ChunkRegs& cr) {
    static_assert(!ONEHOT || KC == 32, "one-hot jobs use the swizzled 32-state chunks");
    if (n > 0) gather_job<NP, KC, ONEHOT>(cr, jobs[0], xs, Sg);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i >= n) break;
        pipe_drain(sm, pp);   // chunk buffer free
        if (ONEHOT && jobs[i].st) onehot_row_sw(sm.a_hi, cr.s, jobs[i].q, S);
        else scatter_any<kTM, KC, NP>(cr.a, sm.a_hi, sm.a_lo, Sg, jobs[i].q);
        scatter_any<NP, KC, NP>(cr.b, sm.b_hi, sm.b_lo, Sg, jobs[i].q);
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0)
            issue_chunk<KC>(sm, tmem + jobs[i].col, NP, jobs[i].q == 0,
                            ONEHOT && jobs[i].st != nullptr, chunk_pieces<NP>(Sg, jobs[i].q) / 2);
        pp.pending = true;
        if (i + 1 < n) gather_job<NP, KC, ONEHOT>(cr, jobs[i + 1], xs, Sg);
    }
}

// Columns [col + 16 j, col + 16 j + 16) of this thread's TMEM lane.
__device__ __forceinline__ void tmem_chunk(uint32_t tmem, int col, int j, float y[16]) {
    tmem_ld16(tmem + ((uint32_t)(threadIdx.x & ~31) << 16) + (uint32_t)(col + 16 * j), y);
}

// y[q] = M[16 j + q][s] for a compact tip state s (the pad value for the
// missing state, zero for states >= S), read from the transposed image: row s
// of M^T is column s of M.
__device__ __forceinline__ void tip_chunk(const float* mt, int s, int S, int Sg, float pad, int j,
                                          float y[16]) {
    const bool ok = s >= 0 && s < S;
    const float* row = mt + (size_t)(ok ? s : 0) * Sg + 16 * j;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        if (16 * j + 4 * k < Sg) ldg4(row + 4 * k, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int i = 16 * j + 4 * k + q;
            y[4 * k + q] = i < S ? (ok ? v[q] : pad) : 0.f;
        }
    }
}

// out[16 j + q] *= operand chunk j, for all chunks, from TMEM columns
// [col, col + NP) for partials and for one-hot tip rows alike; a missing tip
// state takes the matrix's pad value (zero for states >= S).
template <int NP>
__device__ __forceinline__ void mul_operand_oh(float out[NP], bool states, uint32_t tmem, int col,
                                               int s, int S, float pad) {
    const bool miss = states && (s < 0 || s >= S);
#pragma unroll
    for (int j = 0; j < NP / 16; ++j) {
        float y[16];
        tmem_chunk(tmem, col, j, y);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int i = 16 * j + q;
            out[i] *= miss ? (i < S ? pad : 0.f) : y[q];
        }
    }
}

// out[16 j + q] *= operand chunk j, for all chunks: the operand comes from
// TMEM columns [col, col + NP) or, for a tip child, from the matrix image.
template <int NP>
__device__ __forceinline__ void mul_operand(float out[NP], bool states, uint32_t tmem, int col,
                                            const float* mt, int s, int S, int Sg, float pad) {
#pragma unroll
    for (int j = 0; j < NP / 16; ++j) {
        float y[16];
        if (states) tip_chunk(mt, s, S, Sg, pad, j, y);
        else tmem_chunk(tmem, col, j, y);
#pragma unroll
        for (int q = 0; q < 16; ++q) out[16 * j + q] *= y[q];
    }
}

// Cluster exchanges: entry i of every CTA's shared array, the C <= 8 remote
// loads issued together (a loop bounded by the run-time C would wait for each
// load before the next), then combined in rank order.
__device__ __forceinline__ float cluster_max(cg::cluster_group& cl, float* a, int i, int C) {
    float u[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) u[r] = r < C ? cl.map_shared_rank(a, r < C ? r : 0)[i] : 0.f;
    float m = 0.f;
#pragma unroll
    for (int r = 0; r < 8; ++r) m = u[r] > m ? u[r] : m;
    return m;
}

// Sums over the cluster's CTAs of entries 2 i and 2 i + 1, in rank order.
__device__ __forceinline__ void cluster_sum2(cg::cluster_group& cl, double* a, int i, int C,
                                             double& s0, double& s1) {
    double u[8], v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const double* rem = cl.map_shared_rank(a, r < C ? r : 0);
        u[r] = r < C ? rem[2 * i] : 0.0;
        v[r] = r < C ? rem[2 * i + 1] : 0.0;
    }
    s0 = 0;
    s1 = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        if (r < C) {
            s0 += u[r];
            s1 += v[r];
        }
    }
}

// Rescale (cluster-wide maximum over categories and states < S) or fixed
// scaling, then store row t of the tile.  Same arithmetic as finish_tile in
// k_generic.cu.
//
// The maximum is exchanged through sm.smax, whose two halves alternate per
// rescaling (`nresc` counts them): a CTA writes a half again only after the
// next rescaling's cluster barrier, which every CTA of the cluster reaches
// after reading that half, so one barrier per rescaling suffices.  The walk
// ends with a cluster barrier, so no CTA exits while another reads its smax.
// Rows read through the same staging tiles: load_tile_sw issues the
// coalesced loads of rows p0 .. p0 + 127 of category c into registers (lane
// mapping of gather_sw, 4 whole rows per warp instruction; states >= Sg are
// zero), stage_tile_sw writes them to the staging tiles once those are free,
// and after a barrier row_from_stage gives each thread its own row.
template <int NP>
__device__ __forceinline__ void load_tile_sw(float v[][4], const float* src, int p0, int c,
                                             int C, int Sg) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = warp * 4 + (lane >> 3), k8 = lane & 7;
#pragma unroll
    for (int h = 0; h < (NP + 31) / 32; ++h) {
        const int col = 32 * h + 4 * k8;
#pragma unroll
        for (int i = 0; i < kTM / 16; ++i) {
            float* d = v[h * (kTM / 16) + i];
            d[0] = d[1] = d[2] = d[3] = 0.f;
            if (col < Sg) ld4(src + ((size_t)(p0 + r0 + 16 * i) * C + c) * Sg + col, d);
        }
    }
}

template <int NP, typename SM>
__device__ __forceinline__ void stage_tile_sw(SM& sm, const float v[][4]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = warp * 4 + (lane >> 3), k8 = lane & 7;
#pragma unroll
    for (int h = 0; h < (NP + 31) / 32; ++h) {
        float* half = h == 0 ? sm.a_hi : sm.a_lo;
#pragma unroll
        for (int i = 0; i < kTM / 16; ++i) {
            const int r = r0 + 16 * i;
            st4(half + r * 32 + ((k8 ^ (r & 7)) * 4), v[h * (kTM / 16) + i]);
        }
    }
}

template <int NP, typename SM>
__device__ __forceinline__ void row_from_stage(SM& sm, float z[NP]) {
    const int t = threadIdx.x;
#pragma unroll
    for (int kc = 0; kc < NP / 4; ++kc) {
        const float* half = kc < 8 ? sm.a_hi : sm.a_lo;
        ld4(half + t * 32 + (((kc & 7) ^ (t & 7)) * 4), z + 4 * kc);
    }
}

// A tile of rows stored through the swizzled staging tiles (sm.a_hi: states
// 0-31, sm.a_lo: 32-63; free once the op's MMAs have completed): each thread
// writes its row, then every warp stores 4 whole rows (128 contiguous bytes
// each) per instruction, instead of 32 rows 16 bytes apiece.  Rows outside the
// op's pattern range are not stored.  Ends with the staging tiles still in
// use by the stores' reads: the caller's barrier before the next op's chunk
// writes covers them.
template <int NP, typename SM>
__device__ __forceinline__ void store_tile_sw(SM& sm, const OpDesc& op, const float out[NP],
                                              int p0, int c, int C, int Sg) {
    const int t = threadIdx.x;
#pragma unroll
    for (int kc = 0; kc < NP / 4; ++kc) {
        float* half = kc < 8 ? sm.a_hi : sm.a_lo;
        st4(half + t * 32 + (((kc & 7) ^ (t & 7)) * 4), out + 4 * kc);
    }
    __syncthreads();
    const int warp = t >> 5, lane = t & 31;
    const int r0 = warp * 4 + (lane >> 3), k8 = lane & 7;
    float* dest = static_cast<float*>(op.dest);
#pragma unroll
    for (int h = 0; h < (NP + 31) / 32; ++h) {
        const float* half = h == 0 ? sm.a_hi : sm.a_lo;
        const int col = 32 * h + 4 * k8;
        if (col >= Sg) continue;
#pragma unroll
        for (int i = 0; i < kTM / 16; ++i) {
            const int r = r0 + 16 * i;
            const int p = p0 + r;
            if (p < op.p_begin || p >= op.p_end) continue;
            float v[4];
            ld4(half + r * 32 + ((k8 ^ (r & 7)) * 4), v);
            st4(dest + ((size_t)p * C + c) * Sg + col, v);
        }
    }
}

template <int NP, typename SM, bool STORE = true>
__device__ __forceinline__ void finish_row(SM& sm, const OpDesc& op, float out[NP], int p,
                                           int c, int C, int S, int Sg, double* cum,
                                           int log_scalers, int& nresc) {
    const bool mine = p >= op.p_begin && p < op.p_end;   // the op's pattern range
    if (op.cum) cum = op.cum;
    if (op.scale_write) {
        // maximum over states < S as a pairwise tree (6 dependent steps for
        // 64 states instead of a 64-step chain); the same value.  Step h
        // folds entry i + h into entry i for every i that is a multiple of
        // 2h, which covers any NP (48 included), not only powers of two.
        float mx[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) mx[i] = (i < S && out[i] > 0.f) ? out[i] : 0.f;
#pragma unroll
        for (int h = 1; h < NP; h <<= 1)
#pragma unroll
            for (int i = 0; i + h < NP; i += 2 * h)
                mx[i] = mx[i + h] > mx[i] ? mx[i + h] : mx[i];
        float m = mx[0];
        float* sx = sm.smax + (nresc & 1) * kTM;
        ++nresc;
        sx[threadIdx.x] = m;
        cg::cluster_group cluster = cg::this_cluster();
        cluster.sync();
        m = cluster_max(cluster, sx, threadIdx.x, C);
        if (m == 0.f) m = 1.f;
        const float inv = recip(m);
#pragma unroll
        for (int i = 0; i < NP; ++i) out[i] *= inv;
        if (c == 0 && mine) {
            const double lm = scale_log(m);
            op.scale_write[p] = log_scalers ? lm : (double)m;
            if (cum) cum[p] += lm;
        }
    } else if (op.scale_read) {
        const float inv = recip((float)op.scale_read[p]);
#pragma unroll
        for (int i = 0; i < NP; ++i) out[i] *= inv;
    }
    if (!STORE || !mine) return;
    float* d = static_cast<float*>(op.dest) + ((size_t)p * C + c) * Sg;
#pragma unroll
    for (int j = 0; j < NP / 4; ++j)
        if (4 * j < Sg) st4(d + 4 * j, out + 4 * j);
}

// At least 3 resident CTAs per SM (<= 170 registers a thread): with 316-CTA
// grids of 10k-pattern, 4-category data that keeps a launch in one wave.
// Segment of a batched launch holding pattern tile q (segs sorted by first_cta,
// which counts tiles for the tensor-core kernels).
template <typename Seg>
__device__ __forceinline__ int tc_find_seg(const Seg* segs, int nseg, int q) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].first_cta <= q) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// BATCH: a launch over several instances with the same S and C (segs); tile
// q of the grid belongs to the segment whose tiles hold it, and that
// segment's op list, cumulative buffer and scaler kind replace the arguments.
// A batched launch of 32 or fewer states runs many waves of CTAs, so it takes
// 4 CTAs per SM (128 registers): each chain runs a little slower, the SM
// holds a third more of them (batch256: +2.5 %).  One instance's launch
// keeps 3, which fit its grid in fewer waves (amino acid, 20k patterns:
// 4 per SM was slower).
template <int NP, int KC, bool PRE, bool BATCH>
__global__ void __launch_bounds__(kTT, (BATCH && NP <= 32) ? 4 : 3)
k_walk_tc(const OpDesc* __restrict__ ops, int nops, int S, int Sg, int C, double* cum,
          int log_scalers, const WalkSeg* __restrict__ segs, int nseg) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // tiles on 1024-byte boundaries (the swizzle's period; launches add 1 KB)
    TcSmem& sm = *reinterpret_cast<TcSmem*>(
        smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
    using G = TcGeo<NP>;
    const int t = threadIdx.x;
    const int c = blockIdx.x % C;
    int q = blockIdx.x / C;
    // BATCH: the CTA's segment lives in shared memory and its op list,
    // cumulative buffer and scaler kind are read where they are used, instead
    // of occupying registers for the whole walk
    __shared__ WalkSeg s_sg;
    if constexpr (BATCH) {
        if (t == 0) s_sg = segs[tc_find_seg(segs, nseg, q)];
        __syncthreads();
        nops = s_sg.nops;
        q -= s_sg.first_cta;
    }
    const int p0 = q * kTM;
    const int p = p0 + t;
    constexpr int NKC = chunks_of<NP>();
    const size_t xs = (size_t)C * Sg;            // partials row stride (elements)
    const size_t mo = (size_t)c * Sg * Sg;       // category offset in a matrix

    if (t == 0) {
        mbar_init(&sm.bar, 1);
        mbar_init_fence();
    }
    if (t < 32) {
        tmem_alloc(&sm.tmem, G::TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem;
    Pipe pp;

    ChunkRegs cr;
    int nresc = 0;
    for (int o = 0; o < nops; ++o) {
        const OpDesc& op = (BATCH ? s_sg.ops : ops)[o];
        const bool st1 = !PRE && (op.kind & kX1States), st2 = op.kind & kX2States;
        const float* x1 = static_cast<const float*>(op.x1);
        const float* x2 = static_cast<const float*>(op.x2);
        Job jobs[4];
        int nj = 0;
        float out[NP];
        if (!PRE) {
            // child 1 -> columns [0, NP), child 2 -> [NP, 2 NP)
            // (32-state chunks: a tip child is a one-hot job too)
            for (int q = 0; q < NKC; ++q) {
                if (!st1 || KC == 32)
                    jobs[nj++] = Job{st1 ? nullptr : x1 + (size_t)p0 * xs + (size_t)c * Sg,
                                     static_cast<const float*>(op.m1) + mo,
                                     st1 ? static_cast<const int*>(op.x1) + p0 : nullptr, 0u, q};
            }
            for (int q = 0; q < NKC; ++q) {
                if (!st2 || KC == 32)
                    jobs[nj++] = Job{st2 ? nullptr : x2 + (size_t)p0 * xs + (size_t)c * Sg,
                                     static_cast<const float*>(op.m2) + mo,
                                     st2 ? static_cast<const int*>(op.x2) + p0 : nullptr,
                                     (uint32_t)NP, q};
            }
            run_jobs<NP, KC, KC == 32>(sm, pp, tmem, jobs, nj, xs, Sg, S, cr);
            int s1 = 0, s2 = 0;
            if (st1) s1 = static_cast<const int*>(op.x1)[p];
            if (st2) s2 = static_cast<const int*>(op.x2)[p];
            pipe_drain(sm, pp);
            tc_fence_after();
#pragma unroll
            for (int i = 0; i < NP; ++i) out[i] = 1.f;
            if constexpr (KC == 32) {
                mul_operand_oh<NP>(out, st1, tmem, 0, s1, S, (float)op.pad1);
                mul_operand_oh<NP>(out, st2, tmem, NP, s2, S, (float)op.pad2);
            } else {
                mul_operand<NP>(out, st1, tmem, 0, static_cast<const float*>(op.m1t) + mo, s1, S,
                                Sg, (float)op.pad1);
                mul_operand<NP>(out, st2, tmem, NP, static_cast<const float*>(op.m2t) + mo, s2, S,
                                Sg, (float)op.pad2);
            }
        } else {
            // GEMM 1: (P_sib . x_sib) -> columns [0, NP); a tip sibling's
            // operand is read from the matrix image in the epilogue (one-hot
            // jobs here would cost the walk registers it does not have)
            for (int q = 0; q < NKC; ++q) {
                if (!st2) jobs[nj++] = Job{x2 + (size_t)p0 * xs + (size_t)c * Sg,
                                           static_cast<const float*>(op.m2) + mo, nullptr, 0u, q};
            }
            run_jobs<NP, KC>(sm, pp, tmem, jobs, nj, xs, Sg, S, cr);
            // While GEMM 1 runs: the parent row, the sibling's tip state and the
            // first B chunk of GEMM 2 (rows of P_node^T).
            const float* mt =
                static_cast<const float*>((op.kind & kM1Transposed) ? op.m1 : op.m1t) + mo;
            float par[NP];
            if constexpr (KC == 32) {
                // the parent tile by coalesced loads, through the staging
                // tiles once GEMM 1 has read them
                float v[2 * kTM / 16][4];
                load_tile_sw<NP>(v, x1, p0, c, C, Sg);
                gather_any<NP, KC, true, NP>(cr.b, mt, Sg, Sg, 0, Sg);
                pipe_drain(sm, pp);
                stage_tile_sw<NP>(sm, v);
                __syncthreads();
                row_from_stage<NP>(sm, par);
            } else {
                const float* pr = x1 + ((size_t)p * C + c) * Sg;
#pragma unroll
                for (int j = 0; j < NP / 4; ++j) {
                    par[4 * j] = par[4 * j + 1] = par[4 * j + 2] = par[4 * j + 3] = 0.f;
                    if (4 * j < Sg) ld4(pr + 4 * j, par + 4 * j);
                }
                gather_any<NP, KC, true, NP>(cr.b, mt, Sg, Sg, 0, Sg);
                pipe_drain(sm, pp);
            }
            int s2 = 0;
            if (st2) s2 = static_cast<const int*>(op.x2)[p];
            tc_fence_after();
            // z = pre_parent (.) y, in place; states >= Sg stay zero (K padding)
            float* z = par;
            mul_operand<NP>(z, st2, tmem, 0, static_cast<const float*>(op.m2t) + mo, s2, S, Sg,
                            (float)op.pad2);
            // GEMM 2: dest = z . P_node -> columns [NP, 2 NP)
            for (int q = 0; q < NKC; ++q) {
                pipe_drain(sm, pp);
                if constexpr (KC == 32) {
                    if (q == 0) store_row_sw128<NP, 0>(sm.a_hi, sm.a_lo, z);
                    else store_row_sw128<NP, 1>(sm.a_hi, sm.a_lo, z);
                } else {
                    if (q == 0) store_row<NP, KC, 0>(sm.a_hi, sm.a_lo, z);
                    else store_row<NP, KC, 1>(sm.a_hi, sm.a_lo, z);
                }
                scatter_any<NP, KC, NP>(cr.b, sm.b_hi, sm.b_lo, Sg, q);
                fence_async_smem();
                tc_fence_before();
                __syncthreads();
                if (t == 0)
                    issue_chunk<KC>(sm, tmem + NP, NP, q == 0, false, chunk_pieces<NP>(Sg, q) / 2);
                pp.pending = true;
                if (q + 1 < NKC) gather_any<NP, KC, true, NP>(cr.b, mt, Sg, Sg, (q + 1) * KC, Sg);
            }
            pipe_drain(sm, pp);
            tc_fence_after();
#pragma unroll
            for (int j = 0; j < NP / 16; ++j) tmem_chunk(tmem, NP, j, out + 16 * j);
        }
        double* const cum_o = PRE ? nullptr : (BATCH ? s_sg.cum : cum);
        const int ls_o = BATCH ? s_sg.log_scalers : log_scalers;
        if constexpr (KC == 32) {
            finish_row<NP, TcSmem, false>(sm, op, out, p, c, C, S, Sg, cum_o, ls_o, nresc);
            store_tile_sw<NP>(sm, op, out, p0, c, C, Sg);
        } else {
            finish_row<NP>(sm, op, out, p, c, C, S, Sg, cum_o, ls_o, nresc);
        }
        // TMEM reads of this op done before the next op's MMAs overwrite them;
        // this op's stores visible to the CTA before the next op's loads.
        tc_fence_before();
        __syncthreads();
    }
    pipe_drain(sm, pp);
    tc_fence_after();
    cg::this_cluster().sync();   // every remote read of this CTA's smax is done
    if (t < 32) tmem_dealloc(tmem, G::TCOLS);
}

// ------------------------------------------------ TMA-fed walk (variant 2)
// The walk of k_walk_tc with every contraction chunk brought into shared
// memory by TMA (cp.async.bulk.tensor) in the 128-byte swizzled K-major
// layout that the MMA reads directly.
//
// K is cut into chunks of 32 states, one 128-byte row per pattern (A: box
// {32, 1, 128} of the [Pp][C][Sg] partials) and per matrix row (B: box
// {32, NP, 1} of [C][Sg][Sg]); states and rows past Sg are the tensor map's
// zero fill.  The tensor core reads the top 19 bits of each 32-bit value for
// kind::tf32, so the raw tile is the hi half of the 3 x tf32 split as it
// stands.  Threads only write lo = x - hi (same swizzled positions, so the
// pass is elementwise) for A and B.  Two stages: a chunk's loads fly while the
// previous chunk is split and multiplied.  A stage, and its lo buffer, are
// reused once the MMAs that read them have committed (their mbarrier).  The
// pre-order's second product takes its A rows from registers (z), written
// hi and lo at their swizzled positions.
constexpr int kTK = 32;                          // K states per chunk (128-byte rows)
struct TcTma {
    float ahi[2][kTM * kTK];
    float alo[2][kTM * kTK];
    float bhi[2][64 * kTK];
    float blo[2][64 * kTK];
    float smax[2 * kTM];
    double nd[kTM * 2];
    uint64_t tma_bar[2];
    uint64_t mma_bar[2];
    uint32_t tmem;
};

__device__ __forceinline__ void tma_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Box at (x, y, z) of a 3-D tensor map into shared memory, completing on bar.
__device__ __forceinline__ void tma_load3(void* dst, const TmaMap* map, int x, int y, int z,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}


// lo = x - hi of n floats (multiple of 512) of a tile, elementwise.
__device__ __forceinline__ void write_lo(float* lo, const float* hi, int n) {
    for (int i = threadIdx.x * 4; i < n; i += kTT * 4) {
        const float4 x = *reinterpret_cast<const float4*>(hi + i);
        float4 l;
        float h;
        split_tf32(x.x, h, l.x);
        split_tf32(x.y, h, l.y);
        split_tf32(x.z, h, l.z);
        split_tf32(x.w, h, l.w);
        *reinterpret_cast<float4*>(lo + i) = l;
    }
}

// Row t (this thread's) of an A tile from registers: z[Q kTK + k], hi and lo,
// at the swizzled positions (16-byte piece kc of row t at kc ^ (t & 7)).
template <int NP, int Q>
__device__ __forceinline__ void store_row_sw(float* hi, float* lo, const float z[NP]) {
    const int t = threadIdx.x;
#pragma unroll
    for (int kc = 0; kc < kTK / 4; ++kc) {
        float h4[4], l4[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = Q * kTK + kc * 4 + q;
            split_tf32(k < NP ? z[k < NP ? k : 0] : 0.f, h4[q], l4[q]);
        }
        const int off = t * kTK + ((kc ^ (t & 7)) * 4);
        st4(hi + off, h4);
        st4(lo + off, l4);
    }
}

// The MMAs of one chunk (thread 0): 4 K steps of 8, hi.hi + hi.lo + lo.hi,
// committed to the stage's mbarrier.
template <int NP>
__device__ __forceinline__ void issue_chunk_sw(TcTma& sm, int s, uint32_t d_tmem, bool first) {
    const uint32_t idesc = idesc_tf32(kTM, NP);
    const uint32_t ah = smem_u32(sm.ahi[s]), al = smem_u32(sm.alo[s]);
    const uint32_t bh = smem_u32(sm.bhi[s]), bl = smem_u32(sm.blo[s]);
    tc_fence_after();
#pragma unroll
    for (int k = 0; k < kTK / 8; ++k) {
        const uint32_t o = (uint32_t)k * 32u;
        const uint64_t dah = smem_desc_sw128(ah + o), dal = smem_desc_sw128(al + o);
        const uint64_t dbh = smem_desc_sw128(bh + o), dbl = smem_desc_sw128(bl + o);
        mma_tf32(d_tmem, dah, dbh, idesc, (first && k == 0) ? 0u : 1u);
        mma_tf32(d_tmem, dah, dbl, idesc, 1u);
        mma_tf32(d_tmem, dal, dbh, idesc, 1u);
    }
    mma_commit(&sm.mma_bar[s]);
}

// Chunk pipeline state: chunks are numbered over the whole walk; chunk g uses
// stage g & 1.  Phases of each stage's two barriers, and whether an MMA
// commit on a stage is still unwaited.
struct TmaPipe {
    uint32_t tphase[2] = {0, 0};
    uint32_t mphase[2] = {0, 0};
    bool mpending[2] = {false, false};
    bool failed = false;
    int g = 0;
};

__device__ __forceinline__ void mma_wait_stage(TcTma& sm, TmaPipe& tp, int s) {
    if (tp.mpending[s]) {
        mbar_wait(&sm.mma_bar[s], tp.mphase[s], tp.failed);
        tp.mphase[s] ^= 1u;
        tp.mpending[s] = false;
    }
}

// One chunk job: A from a tensor map (a != null) or from registers, B from a
// tensor map.
struct TmaJob {
    const TmaMap* a;
    const TmaMap* b;
    uint32_t col;       // TMEM accumulator column
    int q;              // K chunk
};

// Thread 0: load job j's tiles into stage s.  Every thread has waited, just
// before, for the MMAs that last read the stage (mma_wait_stage), so that all
// threads keep the same barrier phases.
template <int NP>
__device__ __forceinline__ void tma_issue(TcTma& sm, int s, const TmaJob& j, int c, int p0) {
    if (!j.b) {
        // no tensor map: report it, and complete the stage's phase without
        // loading so that no wait runs out
        atomicExch(&b200_tc_status, 1);
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&sm.tma_bar[s]))
                     : "memory");
        return;
    }
    const uint32_t bytes = (uint32_t)((j.a ? kTM : 0) + NP) * kTK * 4;
    tma_expect(&sm.tma_bar[s], bytes);
    if (j.a) tma_load3(sm.ahi[s], j.a, j.q * kTK, c, p0, &sm.tma_bar[s]);
    tma_load3(sm.bhi[s], j.b, j.q * kTK, 0, c, &sm.tma_bar[s]);
}

// Run n chunk jobs (A from tensor maps); job i + 1's loads are issued before
// job i is split and multiplied.
template <int NP>
__device__ __forceinline__ void run_jobs_sw(TcTma& sm, TmaPipe& tp, uint32_t tmem,
                                            const TmaJob (&jobs)[4], int n, int c, int p0) {
    if (n > 0) {
        mma_wait_stage(sm, tp, tp.g & 1);
        if (threadIdx.x == 0) tma_issue<NP>(sm, tp.g & 1, jobs[0], c, p0);
    }
    for (int i = 0; i < n; ++i) {
        const int s = (tp.g + i) & 1;
        if (i + 1 < n) {
            mma_wait_stage(sm, tp, s ^ 1);
            if (threadIdx.x == 0) tma_issue<NP>(sm, s ^ 1, jobs[i + 1], c, p0);
        }
        mbar_wait(&sm.tma_bar[s], tp.tphase[s], tp.failed);
        tp.tphase[s] ^= 1u;
        write_lo(sm.alo[s], sm.ahi[s], kTM * kTK);
        write_lo(sm.blo[s], sm.bhi[s], NP * kTK);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (threadIdx.x == 0) issue_chunk_sw<NP>(sm, s, tmem + jobs[i].col, jobs[i].q == 0);
        tp.mpending[s] = true;
    }
    tp.g += n;
}

// Wait for every committed MMA (both stages).
__device__ __forceinline__ void mma_drain(TcTma& sm, TmaPipe& tp) {
    mma_wait_stage(sm, tp, 0);
    mma_wait_stage(sm, tp, 1);
}

template <int NP, bool PRE>
__global__ void __launch_bounds__(kTT, 2)
k_walk_tc_tma(const OpDesc* __restrict__ ops, const TcOpMaps* __restrict__ maps, int nops,
              int S, int Sg, int C, double* cum, int log_scalers) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // tiles at a 1024-byte aligned shared address (the swizzle's period; the
    // launch adds 1 KB of slack)
    unsigned char* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    TcTma& sm = *reinterpret_cast<TcTma*>(base);
    using G = TcGeo<NP>;
    const int t = threadIdx.x;
    const int c = blockIdx.x % C;
    const int p0 = (blockIdx.x / C) * kTM;
    const int p = p0 + t;
    constexpr int NKC = NP > kTK ? 2 : 1;
    const size_t mo = (size_t)c * Sg * Sg;

    if (t == 0) {
        for (int k = 0; k < 2; ++k) {
            mbar_init(&sm.tma_bar[k], 1);
            mbar_init(&sm.mma_bar[k], 1);
        }
        mbar_init_fence();
    }
    if (t < 32) {
        tmem_alloc(&sm.tmem, G::TCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem;
    TmaPipe tp;
    int nresc = 0;
    for (int o = 0; o < nops; ++o) {
        const OpDesc& op = ops[o];
        const TcOpMaps mp = maps[o];
        const bool st1 = !PRE && (op.kind & kX1States), st2 = op.kind & kX2States;
        TmaJob jobs[4];
        int nj = 0;
        float out[NP];
        if (!PRE) {
            // child 1 -> columns [0, NP), child 2 -> [NP, 2 NP)
            for (int q = 0; q < NKC; ++q)
                if (!st1) jobs[nj++] = TmaJob{mp.a1, mp.b1, 0u, q};
            for (int q = 0; q < NKC; ++q)
                if (!st2) jobs[nj++] = TmaJob{mp.a2, mp.b2, (uint32_t)NP, q};
            run_jobs_sw<NP>(sm, tp, tmem, jobs, nj, c, p0);
            int s1 = 0, s2 = 0;
            if (st1) s1 = static_cast<const int*>(op.x1)[p];
            if (st2) s2 = static_cast<const int*>(op.x2)[p];
            mma_drain(sm, tp);
            tc_fence_after();
#pragma unroll
            for (int i = 0; i < NP; ++i) out[i] = 1.f;
            mul_operand<NP>(out, st1, tmem, 0, static_cast<const float*>(op.m1t) + mo, s1, S, Sg,
                            (float)op.pad1);
            mul_operand<NP>(out, st2, tmem, NP, static_cast<const float*>(op.m2t) + mo, s2, S, Sg,
                            (float)op.pad2);
        } else {
            // GEMM 1: (P_sib . x_sib) -> columns [0, NP)
            for (int q = 0; q < NKC; ++q)
                if (!st2) jobs[nj++] = TmaJob{mp.a2, mp.b2, 0u, q};
            run_jobs_sw<NP>(sm, tp, tmem, jobs, nj, c, p0);
            float par[NP];
            {
                const float* pr = static_cast<const float*>(op.x1) + ((size_t)p * C + c) * Sg;
#pragma unroll
                for (int j = 0; j < NP / 4; ++j) {
                    par[4 * j] = par[4 * j + 1] = par[4 * j + 2] = par[4 * j + 3] = 0.f;
                    if (4 * j < Sg) ld4(pr + 4 * j, par + 4 * j);
                }
            }
            int s2 = 0;
            if (st2) s2 = static_cast<const int*>(op.x2)[p];
            // GEMM 2's first B chunk (rows of P_node^T) while GEMM 1 runs
            const TmaJob j0{nullptr, mp.b1, (uint32_t)NP, 0};
            mma_wait_stage(sm, tp, tp.g & 1);
            if (t == 0) tma_issue<NP>(sm, tp.g & 1, j0, c, p0);
            mma_drain(sm, tp);
            tc_fence_after();
            float* z = par;
            mul_operand<NP>(z, st2, tmem, 0, static_cast<const float*>(op.m2t) + mo, s2, S, Sg,
                            (float)op.pad2);
            // GEMM 2: dest = z . P_node -> columns [NP, 2 NP); A rows from z
#pragma unroll
            for (int q = 0; q < NKC; ++q) {
                const int s = tp.g & 1;
                if (q + 1 < NKC) {
                    mma_wait_stage(sm, tp, s ^ 1);
                    if (t == 0)
                        tma_issue<NP>(sm, s ^ 1, TmaJob{nullptr, mp.b1, (uint32_t)NP, q + 1}, c,
                                      p0);
                }
                if (q == 0) store_row_sw<NP, 0>(sm.ahi[s], sm.alo[s], z);
                else store_row_sw<NP, 1>(sm.ahi[s], sm.alo[s], z);
                mbar_wait(&sm.tma_bar[s], tp.tphase[s], tp.failed);
                tp.tphase[s] ^= 1u;
                write_lo(sm.blo[s], sm.bhi[s], NP * kTK);
                fence_async_smem();
                tc_fence_before();
                __syncthreads();
                if (t == 0) issue_chunk_sw<NP>(sm, s, tmem + NP, q == 0);
                tp.mpending[s] = true;
                ++tp.g;
            }
            mma_drain(sm, tp);
            tc_fence_after();
#pragma unroll
            for (int j = 0; j < NP / 16; ++j) tmem_chunk(tmem, NP, j, out + 16 * j);
        }
        finish_row<NP>(sm, op, out, p, c, C, S, Sg, PRE ? nullptr : cum, log_scalers, nresc);
        tc_fence_before();
        __syncthreads();
    }
    mma_drain(sm, tp);
    tc_fence_after();
    cg::this_cluster().sync();   // every remote read of this CTA's smax is done
    if (t < 32) tmem_dealloc(tmem, G::TCOLS);
}

// Edge derivatives: cluster = (pattern tile, branch), CTA = category (the
// decomposition of k_deriv_x in k_generic.cu).  Y = post . D^T on the tensor
// cores; num / den per category in FP32, combined over categories in FP64.
// BATCH: a launch over several instances (same S and C); cluster q belongs to the
// segment whose (branch, tile) clusters hold it, and that segment's branches,
// weights, pattern count and block partials replace the arguments.
template <int NP, int KC, bool BATCH>
__global__ void __launch_bounds__(kTT, 3)
k_deriv_tc(const DerivDesc* __restrict__ desc, const double* __restrict__ catw,
           const double* __restrict__ patw, int S, int Sg, int C, int P, int ntiles,
           double* site, double* block, const DerivSeg* __restrict__ segs, int nseg) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // tiles on 1024-byte boundaries (the swizzle's period; launches add 1 KB)
    TcSmem& sm = *reinterpret_cast<TcSmem*>(
        smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
    using G = TcGeo<NP>;
    const int t = threadIdx.x;
    const int c = blockIdx.x % C;
    int q = blockIdx.x / C;
    int nb_all = gridDim.x / (C * ntiles);
    if constexpr (BATCH) {
        const DerivSeg& sg = segs[tc_find_seg(segs, nseg, q)];
        desc = sg.desc;
        catw = sg.catw;
        patw = sg.patw;
        P = sg.P;
        ntiles = sg.nblk;
        block = sg.block;
        site = nullptr;
        nb_all = sg.nb;
        q -= sg.first_cta;
    }
    const int tile = q % ntiles;
    const int b = q / ntiles;
    const int p0 = tile * kTM;
    const int p = p0 + t;
    constexpr int NKC = chunks_of<NP>();
    const size_t xs = (size_t)C * Sg;
    const DerivDesc& dd = desc[b];
    const size_t mo = (size_t)c * Sg * Sg;
    const bool states = dd.post_is_states;

    if (t == 0) {
        mbar_init(&sm.bar, 1);
        mbar_init_fence();
    }
    if (t < 32) {
        tmem_alloc(&sm.tmem, G::DCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem;
    Pipe pp;

    const float* post = static_cast<const float*>(dd.post);
    ChunkRegs cr;
    Job jobs[4];
    int nj = 0;
    for (int q = 0; q < NKC; ++q) {
        if (!states || KC == 32)
            jobs[nj++] = Job{states ? nullptr : post + (size_t)p0 * xs + (size_t)c * Sg,
                             static_cast<const float*>(dd.dmat) + mo,
                             states ? static_cast<const int*>(dd.post) + p0 : nullptr, 0u, q};
    }
    run_jobs<NP, KC, KC == 32>(sm, pp, tmem, jobs, nj, xs, Sg, S, cr);
    // While the MMAs run: this row of the pre-order partials and of the
    // post-order partials (or the tip state).
    const float* pre = static_cast<const float*>(dd.pre) + ((size_t)p * C + c) * Sg;
    const float* xr = post + ((size_t)p * C + c) * Sg;
    float pv[NP], xv[NP];
    int s = 0;
    if (states) s = static_cast<const int*>(dd.post)[p];
#pragma unroll
    for (int j = 0; j < NP / 4; ++j) {
        pv[4 * j] = pv[4 * j + 1] = pv[4 * j + 2] = pv[4 * j + 3] = 0.f;
        xv[4 * j] = xv[4 * j + 1] = xv[4 * j + 2] = xv[4 * j + 3] = 0.f;
        if (4 * j < Sg) {
            ld4(pre + 4 * j, pv + 4 * j);
            if (!states) ld4(xr + 4 * j, xv + 4 * j);
        }
    }
    pipe_drain(sm, pp);
    tc_fence_after();
    // four interleaved partial sums each for n and d (shorter dependent
    // chains), added pairwise at the end
    float nq[4] = {0.f, 0.f, 0.f, 0.f}, dq[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < NP / 16; ++j) {
        float y[16];
        if constexpr (KC == 32) {
            tmem_chunk(tmem, 0, j, y);     // one-hot rows for a tip
            if (states && (s < 0 || s >= S))
#pragma unroll
                for (int q = 0; q < 16; ++q) y[q] = (float)dd.dpad;
        } else if (states) {
            tip_chunk(static_cast<const float*>(dd.dmatt) + mo, s, S, Sg, (float)dd.dpad, j, y);
        } else {
            tmem_chunk(tmem, 0, j, y);
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int i = 16 * j + q;
            if (i >= S) continue;
            const float x = states ? ((s < 0 || s >= S || s == i) ? 1.f : 0.f) : xv[i];
            nq[q & 3] += pv[i] * y[q];
            dq[q & 3] += pv[i] * x;
        }
    }
    const float n = (nq[0] + nq[1]) + (nq[2] + nq[3]);
    const float d = (dq[0] + dq[1]) + (dq[2] + dq[3]);
    const double w = catw[c];
    sm.nd[t * 2 + 0] = w * (double)n;
    sm.nd[t * 2 + 1] = w * (double)d;
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    if (c == 0) {
        double nn, dn;
        cluster_sum2(cluster, sm.nd, t, C, nn, dn);
        double v1 = 0, v2 = 0;
        if (p < P) {
            const double dv = nn / dn;
            if (site) site[(size_t)b * P + p] = dv;
            v1 = dv * patw[p];
            v2 = dv * dv * patw[p];
        }
        // The tile's sums: a shuffle tree inside each warp, then the warps in
        // order (a fixed order, so the result is the same every run).
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v1 += __shfl_xor_sync(0xffffffffu, v1, o);
            v2 += __shfl_xor_sync(0xffffffffu, v2, o);
        }
        if ((t & 31) == 0) {
            sm.red[(t >> 5) * 2 + 0] = v1;
            sm.red[(t >> 5) * 2 + 1] = v2;
        }
        __syncthreads();
        if (t == 0) {
            double t1 = 0, t2 = 0;
            for (int k = 0; k < kTT / 32; ++k) {
                t1 += sm.red[k * 2 + 0];
                t2 += sm.red[k * 2 + 1];
            }
            block[(size_t)b * ntiles + tile] = t1;
            block[(size_t)(nb_all + b) * ntiles + tile] = t2;
        }
    }
    cluster.sync();   // remote reads done before any CTA of the cluster exits
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t < 32) tmem_dealloc(tmem, G::DCOLS);
}

// ------------------------------------ fused pre-order walk + derivatives
// The pre-order walk of k_walk_tc with each branch's edge derivative taken
// from the registers of its new row (the S > 4 counterpart of the S = 4
// fused walk in k_fused.cu): per op, three contractions on the tensor cores,
//   GEMM 1: Y1 = sib . P_sib^T                  (TMEM columns [0, NP))
//   GEMM 3: Y3 = post_b . D_b^T                 (columns [NP, 2 NP))
//   GEMM 2: pre_b = (pre_parent o Y1) . P_b     (columns [0, NP) again, once
//                                                Y1 has been read)
// GEMM 3 needs nothing the walk computes, so it is issued with GEMM 1 and its
// loads overlap GEMM 1's; the CTA holds 2 NP columns, as the walk does.  From
// pre_b before rescaling, per category c,
//   n_c = sum_i pre_b[i] Y3[i],   q_c = sum_i pre_b[i] post_b[i],
// are exchanged over the cluster with the rescaling maximum (one cluster
// barrier per op, the exchange buffers alternating by op parity), and
// category 0's CTA forms d_p = sum_c w_c n_c / sum_c w_c q_c, the quantity of
// k_deriv_tc (CPU/BeagleCPUImpl.hpp:1940-2083).  The tile's w_p d_p and
// w_p d_p^2 go to block[op][tile] and block[nsum + op][tile]; launch_final_sum
// adds the tiles in a fixed order.  A separate derivative pass would read
// every pre_b back from memory; here it never leaves the registers.
struct TcFusedSmem {
    float a_hi[kTM * 32];
    float a_lo[kTM * 32];
    float b_hi[64 * 32];
    float b_lo[64 * 32];
    float smax[2][kTM];          // alternating by op parity
    double nd[2][kTM * 2];       // w_c n_c, w_c q_c per row, alternating by op parity
    double red[kTT / 32 * 2];
    uint64_t bar;
    uint32_t tmem;
};

template <int NP>
struct TcFusedGeo {
    static constexpr int COLS = TcGeo<NP>::TCOLS;
};

// BATCH: a launch over several instances with the same S and C (segs): tile
// q of the grid belongs to the segment whose tiles hold it, and that
// segment's lists, weights, pattern count and block partials replace the
// arguments.
template <int NP, int KC, bool BATCH>
__global__ void __launch_bounds__(kTT, 3)
k_prederiv_tc(const OpDesc* __restrict__ ops, const DerivDesc* __restrict__ dds, int nops,
              int nsum, int S, int Sg, int C, int P, const double* __restrict__ catw,
              const double* __restrict__ patw, int log_scalers, double* block,
              const PreDerivSeg* __restrict__ segs, int nseg) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TcFusedSmem& sm = *reinterpret_cast<TcFusedSmem*>(
        smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
    constexpr int COLS = TcFusedGeo<NP>::COLS;
    const int t = threadIdx.x;
    const int c = blockIdx.x % C;
    int tile = blockIdx.x / C;
    int ntiles = gridDim.x / C;
    // BATCH: the CTA's segment lives in shared memory and its fields are read
    // where they are used (as the other form reads its kernel parameters),
    // instead of occupying registers for the whole walk
    __shared__ PreDerivSeg s_sg;
    if constexpr (BATCH) {
        if (t == 0) s_sg = segs[tc_find_seg(segs, nseg, tile)];
        __syncthreads();
        ntiles = s_sg.nblk;
        tile -= s_sg.first_cta;
        nops = s_sg.nops;
    }
#define SEG_(field, arg) (BATCH ? s_sg.field : (arg))
    const int p0 = tile * kTM;
    const int p = p0 + t;
    constexpr int NKC = chunks_of<NP>();
    const size_t xs = (size_t)C * Sg;
    const size_t mo = (size_t)c * Sg * Sg;
    const double wc = SEG_(catw, catw)[c];

    if (t == 0) {
        mbar_init(&sm.bar, 1);
        mbar_init_fence();
    }
    if (t < 32) {
        tmem_alloc(&sm.tmem, COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem;
    Pipe pp;
    ChunkRegs cr;
    cg::cluster_group cluster = cg::this_cluster();
    for (int o = 0; o < nops; ++o) {
        const OpDesc& op = SEG_(ops, ops)[o];
        const DerivDesc& dd = SEG_(dds, dds)[o];
        const bool st2 = op.kind & kX2States;
        const bool pst = dd.post_is_states;
        const float* x2 = static_cast<const float*>(op.x2);
        const float* post = static_cast<const float*>(dd.post);
        // GEMM 1, then GEMM 3 (two calls of at most NKC jobs each: the
        // first gather of GEMM 3 still overlaps GEMM 1's last MMAs, and the
        // shorter job lists keep the walk within its register budget)
        {
            Job jobs[4];
            int nj = 0;
            for (int q = 0; q < NKC; ++q)
                if (!st2) jobs[nj++] = Job{x2 + (size_t)p0 * xs + (size_t)c * Sg,
                                           static_cast<const float*>(op.m2) + mo, nullptr, 0u, q};
            run_jobs<NP, KC>(sm, pp, tmem, jobs, nj, xs, Sg, S, cr);
        }
        {
            Job jobs[4];
            int nj = 0;
            for (int q = 0; q < NKC; ++q)
                if (!pst) jobs[nj++] = Job{post + (size_t)p0 * xs + (size_t)c * Sg,
                                           static_cast<const float*>(dd.dmat) + mo, nullptr,
                                           (uint32_t)NP, q};
            run_jobs<NP, KC>(sm, pp, tmem, jobs, nj, xs, Sg, S, cr);
        }
        // While they run: the parent row, the tip states and GEMM 2's first
        // B chunk (rows of P_node^T).
        const float* mt =
            static_cast<const float*>((op.kind & kM1Transposed) ? op.m1 : op.m1t) + mo;
        float z[NP];
        if constexpr (KC == 32) {
            float v[2 * kTM / 16][4];
            load_tile_sw<NP>(v, static_cast<const float*>(op.x1), p0, c, C, Sg);
            gather_any<NP, KC, true, NP>(cr.b, mt, Sg, Sg, 0, Sg);
            pipe_drain(sm, pp);
            stage_tile_sw<NP>(sm, v);
            __syncthreads();
            row_from_stage<NP>(sm, z);
        } else {
            const float* pr = static_cast<const float*>(op.x1) + ((size_t)p * C + c) * Sg;
#pragma unroll
            for (int j = 0; j < NP / 4; ++j) {
                z[4 * j] = z[4 * j + 1] = z[4 * j + 2] = z[4 * j + 3] = 0.f;
                if (4 * j < Sg) ld4(pr + 4 * j, z + 4 * j);
            }
            gather_any<NP, KC, true, NP>(cr.b, mt, Sg, Sg, 0, Sg);
            pipe_drain(sm, pp);
        }
        const int s2 = st2 ? static_cast<const int*>(op.x2)[p] : 0;
        const int sp = pst ? static_cast<const int*>(dd.post)[p] : 0;
        tc_fence_after();
        mul_operand<NP>(z, st2, tmem, 0, static_cast<const float*>(op.m2t) + mo, s2, S, Sg,
                        (float)op.pad2);
        for (int q = 0; q < NKC; ++q) {
            pipe_drain(sm, pp);
            if constexpr (KC == 32) {
                if (q == 0) store_row_sw128<NP, 0>(sm.a_hi, sm.a_lo, z);
                else store_row_sw128<NP, 1>(sm.a_hi, sm.a_lo, z);
            } else {
                if (q == 0) store_row<NP, KC, 0>(sm.a_hi, sm.a_lo, z);
                else store_row<NP, KC, 1>(sm.a_hi, sm.a_lo, z);
            }
            scatter_any<NP, KC, NP>(cr.b, sm.b_hi, sm.b_lo, Sg, q);
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            if (t == 0)   // over Y1, now read
                issue_chunk<KC>(sm, tmem, NP, q == 0, false, chunk_pieces<NP>(Sg, q) / 2);
            pp.pending = true;
            if (q + 1 < NKC) gather_any<NP, KC, true, NP>(cr.b, mt, Sg, Sg, (q + 1) * KC, Sg);
        }
        if constexpr (KC == 32) {
            // this node's post-order tile by coalesced loads through the
            // staging tiles, free once GEMM 2 has completed (issued before
            // the drain, the loads would need registers the walk does not
            // have)
            float v[2 * kTM / 16][4];
            pipe_drain(sm, pp);
            if (!pst) load_tile_sw<NP>(v, post, p0, c, C, Sg);
            if (!pst) stage_tile_sw<NP>(sm, v);
            __syncthreads();
        } else {
            pipe_drain(sm, pp);
        }
        tc_fence_after();
        float out[NP];
#pragma unroll
        for (int j = 0; j < NP / 16; ++j) tmem_chunk(tmem, 0, j, out + 16 * j);
        // derivative terms of this row and category, from pre_b as computed
        float nq[4] = {0.f, 0.f, 0.f, 0.f}, dq[4] = {0.f, 0.f, 0.f, 0.f};
        float mq[4] = {0.f, 0.f, 0.f, 0.f};       // rescaling maximum, four chains
        const float* xr = post + ((size_t)p * C + c) * Sg;
#pragma unroll
        for (int j = 0; j < NP / 16; ++j) {
            float y[16], x[16];
            if (pst) tip_chunk(static_cast<const float*>(dd.dmatt) + mo, sp, S, Sg,
                               (float)dd.dpad, j, y);
            else tmem_chunk(tmem, NP, j, y);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                x[4 * k] = x[4 * k + 1] = x[4 * k + 2] = x[4 * k + 3] = 0.f;
                if constexpr (KC == 32) {
                    const int kc = 4 * j + k;    // this row's piece, from the staging tiles
                    const float* half = kc < 8 ? sm.a_hi : sm.a_lo;
                    if (!pst && kc < NP / 4)
                        ld4(half + t * 32 + (((kc & 7) ^ (t & 7)) * 4), x + 4 * k);
                } else {
                    if (!pst && 16 * j + 4 * k < Sg) ld4(xr + 16 * j + 4 * k, x + 4 * k);
                }
            }
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int i = 16 * j + q;
                if (i >= S) continue;
                const float xv = pst ? ((sp < 0 || sp >= S || sp == i) ? 1.f : 0.f) : x[q];
                nq[q & 3] += out[i] * y[q];
                dq[q & 3] += out[i] * xv;
                mq[q & 3] = out[i] > mq[q & 3] ? out[i] : mq[q & 3];
            }
        }
        const int par = o & 1;
        sm.nd[par][t * 2 + 0] = wc * (double)((nq[0] + nq[1]) + (nq[2] + nq[3]));
        sm.nd[par][t * 2 + 1] = wc * (double)((dq[0] + dq[1]) + (dq[2] + dq[3]));
        if (op.scale_write) {
            const float m01 = mq[1] > mq[0] ? mq[1] : mq[0];
            const float m23 = mq[3] > mq[2] ? mq[3] : mq[2];
            sm.smax[par][t] = m23 > m01 ? m23 : m01;
        }
        // One barrier per op: every CTA's maximum and derivative terms are
        // written; the halves of parity `par` are rewritten at op o + 2, after
        // the next op's barrier, which every CTA reaches after reading them.
        cluster.sync();
        const bool mine = p >= op.p_begin && p < op.p_end;
        if (op.scale_write) {
            float m = cluster_max(cluster, sm.smax[par], t, C);
            if (m == 0.f) m = 1.f;
            const float inv = recip(m);
#pragma unroll
            for (int i = 0; i < NP; ++i) out[i] *= inv;
            if (c == 0 && mine) {
                const double lm = scale_log(m);
                op.scale_write[p] = SEG_(log_scalers, log_scalers) ? lm : (double)m;
            }
        }
        if constexpr (KC == 32) {
            store_tile_sw<NP>(sm, op, out, p0, c, C, Sg);
        } else if (mine) {
            float* dst = static_cast<float*>(op.dest) + ((size_t)p * C + c) * Sg;
#pragma unroll
            for (int j = 0; j < NP / 4; ++j)
                if (4 * j < Sg) st4(dst + 4 * j, out + 4 * j);
        }
        // op o's derivative sums on the cluster's CTA o mod C (spread over
        // the cluster: the others wait for it at the next barrier)
        if (c == o % C) {
            double nn, dn;
            cluster_sum2(cluster, sm.nd[par], t, C, nn, dn);
            double v1 = 0, v2 = 0;
            if (p < SEG_(P, P)) {
                const double dv = nn / dn;
                const double wp = SEG_(patw, patw)[p];
                v1 = dv * wp;
                v2 = dv * dv * wp;
            }
#pragma unroll
            for (int sh = 16; sh > 0; sh >>= 1) {
                v1 += __shfl_xor_sync(0xffffffffu, v1, sh);
                v2 += __shfl_xor_sync(0xffffffffu, v2, sh);
            }
            if ((t & 31) == 0) {
                sm.red[(t >> 5) * 2 + 0] = v1;
                sm.red[(t >> 5) * 2 + 1] = v2;
            }
            __syncthreads();
            if (t == 0) {
                double t1 = 0, t2 = 0;
                for (int k = 0; k < kTT / 32; ++k) {
                    t1 += sm.red[k * 2 + 0];
                    t2 += sm.red[k * 2 + 1];
                }
                double* blk = SEG_(block, block);
                blk[(size_t)o * ntiles + tile] = t1;
                blk[(size_t)(SEG_(nops, nsum) + o) * ntiles + tile] = t2;
            }
        }
        // TMEM reads of this op done before the next op's MMAs overwrite
        // them; this op's stores visible to the CTA before later loads.
        tc_fence_before();
        __syncthreads();
    }
#undef SEG_
    pipe_drain(sm, pp);
    tc_fence_after();
    cluster.sync();   // every remote read of this CTA's exchange buffers is done
    if (t < 32) tmem_dealloc(tmem, COLS);
}

// ------------------------------------------ tensor-core fused walk, pairs
// k_prederiv_tc for 17 to 32 states (N = K = 32) on lists made only of
// sibling pairs (kPairFirst on every even op; the launcher refuses other
// lists), one pair a step.  Ops a and b share their parent and each is the
// other's sibling, so the four products their GEMM 1 and GEMM 3 make,
//   Y1_a = post_b . P_b^T    Y3_b = post_b . D_b^T    (A tile post_b)
//   Y1_b = post_a . P_a^T    Y3_a = post_a . D_a^T    (A tile post_a),
// come two from each A tile: the tile is gathered and split once and
// multiplied by two matrices staged side by side (B rows 0-31 and 32-63).
// The parent tile is loaded once for both GEMM 2s, both epilogues' post-order
// rows are staged together, and one cluster barrier exchanges both rescaling
// maxima and both ops' derivative terms.  TMEM: four 32-column accumulators
// (Y1_a, Y3_b, Y1_b, Y3_a); GEMM 2 of each op overwrites its Y1.
struct TcPairSmem {
    float a_hi[kTM * 32];
    float a_lo[kTM * 32];
    float b_hi[64 * 32];
    float b_lo[64 * 32];
    float smax[2][2][kTM];        // [step parity][op of the pair]
    double nd[2][2][kTM * 2];     // [step parity][op of the pair]: w_c n_c, w_c q_c per row
    float inv[2][kTM];            // each row's rescaling factor 1 / m, per op of the pair
    double red[kTT / 32 * 2];
    uint64_t bar;
    uint32_t tmem;
};
constexpr int kPairCols = 128;

// Both products of the A tile in shared memory: 3 x tf32 split MMAs into d1
// (B rows 0-31) and d2 (B rows 32-63), N = 32, ksteps K steps, one commit.
__device__ __forceinline__ void issue_dual(TcPairSmem& sm, uint32_t d1, uint32_t d2, int ksteps) {
    const uint32_t idesc = idesc_tf32(kTM, 32);
    const uint32_t ah = smem_u32(sm.a_hi), al = smem_u32(sm.a_lo);
    const uint32_t bh = smem_u32(sm.b_hi), bl = smem_u32(sm.b_lo);
    constexpr uint32_t kB2 = 32u * 128u;     // B rows 32-63: 4 KB in, 1024-byte aligned
    tc_fence_after();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k >= ksteps) break;
        const uint32_t o = (uint32_t)k * 32u;
        const uint64_t dah = smem_desc_sw128(ah + o), dal = smem_desc_sw128(al + o);
        const uint64_t b1h = smem_desc_sw128(bh + o), b1l = smem_desc_sw128(bl + o);
        const uint64_t b2h = smem_desc_sw128(bh + kB2 + o), b2l = smem_desc_sw128(bl + kB2 + o);
        const uint32_t acc = k == 0 ? 0u : 1u;
        mma_tf32(d1, dah, b1h, idesc, acc);
        mma_tf32(d1, dah, b1l, idesc, 1u);
        mma_tf32(d1, dal, b1h, idesc, 1u);
        mma_tf32(d2, dah, b2h, idesc, acc);
        mma_tf32(d2, dah, b2l, idesc, 1u);
        mma_tf32(d2, dal, b2h, idesc, 1u);
    }
    mma_commit(&sm.bar);
}

// Rows p0 .. p0 + 127 of one 32-column half (registers from load_tile_sw)
// into a staging tile, and this thread's row back out of one.
__device__ __forceinline__ void stage_half_sw(float* half, const float v[][4]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = warp * 4 + (lane >> 3), k8 = lane & 7;
#pragma unroll
    for (int i = 0; i < kTM / 16; ++i) {
        const int r = r0 + 16 * i;
        st4(half + r * 32 + ((k8 ^ (r & 7)) * 4), v[i]);
    }
}

// Derivative terms (n, q) and the rescaling maximum of one op's new row
// `out` (32 states): D . post from TMEM column `col` (a tip's column of D
// from the transposed image), the post-order row from the staging tile.
__device__ __forceinline__ void pair_terms(const float out[32], bool pst, int sp,
                                           const DerivDesc& dd, size_t mo, uint32_t tmem,
                                           uint32_t col, const float* stage, int S, int Sg,
                                           float& n, float& q, float& mx) {
    const int t = threadIdx.x;
    float nq[4] = {0.f, 0.f, 0.f, 0.f}, dq[4] = {0.f, 0.f, 0.f, 0.f}, mq[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        float y[16], x[16];
        if (pst) tip_chunk(static_cast<const float*>(dd.dmatt) + mo, sp, S, Sg, (float)dd.dpad, j,
                           y);
        else tmem_chunk(tmem, (int)col, j, y);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            x[4 * k] = x[4 * k + 1] = x[4 * k + 2] = x[4 * k + 3] = 0.f;
            const int kc = 4 * j + k;
            if (!pst) ld4(stage + t * 32 + ((kc ^ (t & 7)) * 4), x + 4 * k);
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int i = 16 * j + e;
            if (i >= S) continue;
            const float xv = pst ? ((sp < 0 || sp >= S || sp == i) ? 1.f : 0.f) : x[e];
            nq[e & 3] += out[i] * y[e];
            dq[e & 3] += out[i] * xv;
            mq[e & 3] = out[i] > mq[e & 3] ? out[i] : mq[e & 3];
        }
    }
    n = (nq[0] + nq[1]) + (nq[2] + nq[3]);
    q = (dq[0] + dq[1]) + (dq[2] + dq[3]);
    const float m01 = mq[1] > mq[0] ? mq[1] : mq[0];
    const float m23 = mq[3] > mq[2] ? mq[3] : mq[2];
    mx = m23 > m01 ? m23 : m01;
}

template <bool BATCH>
__global__ void __launch_bounds__(kTT, 3)
k_prederiv_tc_pairs(const OpDesc* __restrict__ ops, const DerivDesc* __restrict__ dds, int nops,
                    int nsum, int S, int Sg, int C, int P, const double* __restrict__ catw,
                    const double* __restrict__ patw, int log_scalers, double* block,
                    const PreDerivSeg* __restrict__ segs, int nseg) {
    constexpr int NP = 32;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TcPairSmem& sm = *reinterpret_cast<TcPairSmem*>(
        smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
    const int t = threadIdx.x;
    const int c = blockIdx.x % C;
    int tile = blockIdx.x / C;
    int ntiles = gridDim.x / C;
    __shared__ PreDerivSeg s_sg;
    if constexpr (BATCH) {
        if (t == 0) s_sg = segs[tc_find_seg(segs, nseg, tile)];
        __syncthreads();
        ntiles = s_sg.nblk;
        tile -= s_sg.first_cta;
        nops = s_sg.nops;
    }
#define SEG_(field, arg) (BATCH ? s_sg.field : (arg))
    const int p0 = tile * kTM;
    const int p = p0 + t;
    const size_t xs = (size_t)C * Sg;
    const size_t mo = (size_t)c * Sg * Sg;
    const double wc = SEG_(catw, catw)[c];
    const int np = chunk_pieces<NP>(Sg, 0);        // 16-byte pieces of a row the MMAs read
    const int ks = np / 2;
    constexpr uint32_t cY1a = 0, cY3b = 32, cY1b = 64, cY3a = 96;

    if (t == 0) {
        mbar_init(&sm.bar, 1);
        mbar_init_fence();
    }
    if (t < 32) {
        tmem_alloc(&sm.tmem, kPairCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem;
    Pipe pp;
    ChunkRegs cr;
    cg::cluster_group cluster = cg::this_cluster();
    // The weighted derivative of op oo for each of this tile's rows from
    // every category's terms (nd), then the tile's block sums.
    auto emit_sums = [&](int oo, double* nd) {
        double nn, dn;
        cluster_sum2(cluster, nd, t, C, nn, dn);
        double v1 = 0, v2 = 0;
        if (p < SEG_(P, P)) {
            const double dv = nn / dn;
            const double wp = SEG_(patw, patw)[p];
            v1 = dv * wp;
            v2 = dv * dv * wp;
        }
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) {
            v1 += __shfl_xor_sync(0xffffffffu, v1, sh);
            v2 += __shfl_xor_sync(0xffffffffu, v2, sh);
        }
        if ((t & 31) == 0) {
            sm.red[(t >> 5) * 2 + 0] = v1;
            sm.red[(t >> 5) * 2 + 1] = v2;
        }
        __syncthreads();
        if (t == 0) {
            double t1 = 0, t2 = 0;
            for (int k = 0; k < kTT / 32; ++k) {
                t1 += sm.red[k * 2 + 0];
                t2 += sm.red[k * 2 + 1];
            }
            double* blk = SEG_(block, block);
            blk[(size_t)oo * ntiles + tile] = t1;
            blk[(size_t)(SEG_(nops, nsum) + oo) * ntiles + tile] = t2;
        }
        __syncthreads();   // sm.red free for the next use
    };
    for (int o = 0; o + 1 < nops; o += 2) {
        const OpDesc& A = SEG_(ops, ops)[o];
        const OpDesc& B = SEG_(ops, ops)[o + 1];
        const DerivDesc& Ad = SEG_(dds, dds)[o];
        const DerivDesc& Bd = SEG_(dds, dds)[o + 1];
        const bool tb = A.kind & kX2States;       // post_b is tip states (a's sibling)
        const bool ta = B.kind & kX2States;       // post_a is tip states (b's sibling)
        const float* post_b = static_cast<const float*>(A.x2);
        const float* post_a = static_cast<const float*>(B.x2);
        // 1. Y1_a, Y3_b from the A tile post_b; Y1_b, Y3_a from post_a (a tip
        // tile is none: its products are matrix columns, read in place)
        if (!tb) {
            gather_sw<kTM, false>(cr.a, post_b + (size_t)p0 * xs + (size_t)c * Sg, xs, kTM, 0, Sg,
                                  np);
            gather_sw<32, true>(cr.b, static_cast<const float*>(A.m2) + mo, Sg, Sg, 0, Sg, np);
            gather_sw<32, true>(cr.b + 2, static_cast<const float*>(Bd.dmat) + mo, Sg, Sg, 0, Sg,
                                np);
            pipe_drain(sm, pp);
            scatter_sw<kTM>(cr.a, sm.a_hi, sm.a_lo, np);
            scatter_sw<32>(cr.b, sm.b_hi, sm.b_lo, np);
            scatter_sw<32>(cr.b + 2, sm.b_hi + 32 * 32, sm.b_lo + 32 * 32, np);
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            if (t == 0) issue_dual(sm, tmem + cY1a, tmem + cY3b, ks);
            pp.pending = true;
        }
        if (!ta) {
            gather_sw<kTM, false>(cr.a, post_a + (size_t)p0 * xs + (size_t)c * Sg, xs, kTM, 0, Sg,
                                  np);
            gather_sw<32, true>(cr.b, static_cast<const float*>(B.m2) + mo, Sg, Sg, 0, Sg, np);
            gather_sw<32, true>(cr.b + 2, static_cast<const float*>(Ad.dmat) + mo, Sg, Sg, 0, Sg,
                                np);
            pipe_drain(sm, pp);
            scatter_sw<kTM>(cr.a, sm.a_hi, sm.a_lo, np);
            scatter_sw<32>(cr.b, sm.b_hi, sm.b_lo, np);
            scatter_sw<32>(cr.b + 2, sm.b_hi + 32 * 32, sm.b_lo + 32 * 32, np);
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            if (t == 0) issue_dual(sm, tmem + cY1b, tmem + cY3a, ks);
            pp.pending = true;
        }
        // 2. the parent tile through the staging tile once the products have
        // read the A tiles, and GEMM 2a's B rows (P_a^T)
        const float* mta =
            static_cast<const float*>((A.kind & kM1Transposed) ? A.m1 : A.m1t) + mo;
        const float* mtb =
            static_cast<const float*>((B.kind & kM1Transposed) ? B.m1 : B.m1t) + mo;
        float par[NP];
        {
            float v[kTM / 16][4];
            load_tile_sw<NP>(v, static_cast<const float*>(A.x1), p0, c, C, Sg);
            gather_sw<32, true>(cr.b, mta, Sg, Sg, 0, Sg, np);
            pipe_drain(sm, pp);
            stage_half_sw(sm.a_hi, v);
            __syncthreads();
            row_from_stage<NP>(sm, par);
        }
        tc_fence_after();
        const int sb = tb ? static_cast<const int*>(A.x2)[p] : 0;
        const int sa = ta ? static_cast<const int*>(B.x2)[p] : 0;
        // 3. GEMM 2a: out_a = (parent (.) Y1_a) . P_a into Y1_a's columns,
        // then GEMM 2b the same way (its operand formed while 2a runs)
        float z[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) z[i] = par[i];
        mul_operand<NP>(z, tb, tmem, (int)cY1a, static_cast<const float*>(A.m2t) + mo, sb, S, Sg,
                        (float)A.pad2);
        store_row_sw128<NP, 0>(sm.a_hi, sm.a_lo, z);
        scatter_sw<32>(cr.b, sm.b_hi, sm.b_lo, np);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) issue_chunk<32>(sm, tmem + cY1a, NP, true, false, ks);
        pp.pending = true;
#pragma unroll
        for (int i = 0; i < NP; ++i) z[i] = par[i];
        mul_operand<NP>(z, ta, tmem, (int)cY1b, static_cast<const float*>(B.m2t) + mo, sa, S, Sg,
                        (float)B.pad2);
        gather_sw<32, true>(cr.b, mtb, Sg, Sg, 0, Sg, np);
        pipe_drain(sm, pp);
        store_row_sw128<NP, 0>(sm.a_hi, sm.a_lo, z);
        scatter_sw<32>(cr.b, sm.b_hi, sm.b_lo, np);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) issue_chunk<32>(sm, tmem + cY1b, NP, true, false, ks);
        pp.pending = true;
        // 4. both post-order tiles (coalesced), post_a while GEMM 2b runs,
        // staged once it has read the A tile: post_a in a_hi, post_b in a_lo
        {
            float v[kTM / 16][4];
            if (!ta) load_tile_sw<NP>(v, post_a, p0, c, C, Sg);
            pipe_drain(sm, pp);
            if (!ta) stage_half_sw(sm.a_hi, v);
            if (!tb) load_tile_sw<NP>(v, post_b, p0, c, C, Sg);
            if (!tb) stage_half_sw(sm.a_lo, v);
        }
        __syncthreads();
        tc_fence_after();
        // 5. each op's new row: derivative terms and rescaling maximum, then
        // the row itself (unscaled) over this thread's post-order row in the
        // staging tile, which only this thread reads; one exchange for both
        const int par_ = (o >> 1) & 1;
        {
            float out[NP], n, q, mx;
#pragma unroll
            for (int j = 0; j < NP / 16; ++j) tmem_chunk(tmem, (int)cY1a, j, out + 16 * j);
            pair_terms(out, ta, sa, Ad, mo, tmem, cY3a, sm.a_hi, S, Sg, n, q, mx);
            sm.nd[par_][0][t * 2 + 0] = wc * (double)n;
            sm.nd[par_][0][t * 2 + 1] = wc * (double)q;
            sm.smax[par_][0][t] = mx;
#pragma unroll
            for (int kc = 0; kc < 8; ++kc) st4(sm.a_hi + t * 32 + ((kc ^ (t & 7)) * 4), out + 4 * kc);
#pragma unroll
            for (int j = 0; j < NP / 16; ++j) tmem_chunk(tmem, (int)cY1b, j, out + 16 * j);
            pair_terms(out, tb, sb, Bd, mo, tmem, cY3b, sm.a_lo, S, Sg, n, q, mx);
            sm.nd[par_][1][t * 2 + 0] = wc * (double)n;
            sm.nd[par_][1][t * 2 + 1] = wc * (double)q;
            sm.smax[par_][1][t] = mx;
#pragma unroll
            for (int kc = 0; kc < 8; ++kc) st4(sm.a_lo + t * 32 + ((kc ^ (t & 7)) * 4), out + 4 * kc);
        }
        // Exchange halves of parity par_ are rewritten two steps later, after
        // the next step's barrier, which every CTA reaches after reading them.
        cluster.sync();
        const int ls = SEG_(log_scalers, log_scalers);
        {
            float ia = 1.f, ib = 1.f;
            if (A.scale_write) {
                float m = cluster_max(cluster, sm.smax[par_][0], t, C);
                if (m == 0.f) m = 1.f;
                ia = recip(m);
                if (c == 0 && p >= A.p_begin && p < A.p_end) {
                    const double lm = scale_log(m);
                    A.scale_write[p] = ls ? lm : (double)m;
                }
            }
            if (B.scale_write) {
                float m = cluster_max(cluster, sm.smax[par_][1], t, C);
                if (m == 0.f) m = 1.f;
                ib = recip(m);
                if (c == 0 && p >= B.p_begin && p < B.p_end) {
                    const double lm = scale_log(m);
                    B.scale_write[p] = ls ? lm : (double)m;
                }
            }
            sm.inv[0][t] = ia;
            sm.inv[1][t] = ib;
        }
        __syncthreads();
        // 6. both new tiles out in whole-row stores, each row scaled by its
        // factor on the way
        {
            const int warp = t >> 5, lane = t & 31;
            const int r0 = warp * 4 + (lane >> 3), k8 = lane & 7;
            const int col = 4 * k8;
            if (col < Sg) {
#pragma unroll
                for (int i = 0; i < kTM / 16; ++i) {
                    const int r = r0 + 16 * i;
                    const int pr = p0 + r;
                    float v[4];
                    if (pr >= A.p_begin && pr < A.p_end) {
                        ld4(sm.a_hi + r * 32 + ((k8 ^ (r & 7)) * 4), v);
                        const float f = sm.inv[0][r];
#pragma unroll
                        for (int e = 0; e < 4; ++e) v[e] *= f;
                        st4(static_cast<float*>(A.dest) + ((size_t)pr * C + c) * Sg + col, v);
                    }
                    if (pr >= B.p_begin && pr < B.p_end) {
                        ld4(sm.a_lo + r * 32 + ((k8 ^ (r & 7)) * 4), v);
                        const float f = sm.inv[1][r];
#pragma unroll
                        for (int e = 0; e < 4; ++e) v[e] *= f;
                        st4(static_cast<float*>(B.dest) + ((size_t)pr * C + c) * Sg + col, v);
                    }
                }
            }
        }
        // 7. both ops' derivative sums, op k's on the cluster's CTA k mod C
        // (spread over the cluster: the others wait for it at the next barrier)
        if (c == o % C) emit_sums(o, sm.nd[par_][0]);
        if (c == (o + 1) % C) emit_sums(o + 1, sm.nd[par_][1]);
        // TMEM reads of this step done before the next step's MMAs overwrite
        // them; this step's stores visible to the CTA before later loads.
        tc_fence_before();
        __syncthreads();
    }
#undef SEG_
    pipe_drain(sm, pp);
    tc_fence_after();
    cluster.sync();   // every remote read of this CTA's exchange buffers is done
    if (t < 32) tmem_dealloc(tmem, kPairCols);
}

// Dynamic shared memory of a launch: the struct, raised to the TMEM
// columns' share of the SM's shared memory.  An SM has 228 KB (233,472 B)
// and reserves 1 KB per CTA, so a CTA asking for `cols` of the 512 columns
// takes at least 233,472 * cols / 512 = 456 * cols bytes in all.  Any set of
// CTAs resident on one SM -- of one launch, or of several tensor-core
// launches from different streams or instances -- then holds at most 512
// columns, and a tcgen05.alloc never waits on a CTA that waits on it.
size_t tc_smem(int cols) {
    const size_t need = sizeof(TcSmem) + 1024;   // + alignment slack
    const size_t floor_bytes = (size_t)456 * cols - 1024;
    return need > floor_bytes ? need : floor_bytes;
}

template <typename K, typename... Args>
cudaError_t launch_tc(K kernel, int grid, size_t smem, int cluster, int cols, cudaStream_t s,
                      Args... args) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTT, smem);
    if (e != cudaSuccess) return e;
    if (per_sm * cols > 512) return cudaErrorInvalidConfiguration;   // TMEM could be oversubscribed
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(kTT, 1, 1);
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

template <int NP, int KC>
cudaError_t run_walk_tc(const OpDesc* ops, int nops, bool pre, const Dims& d, double* cum,
                        int ls, cudaStream_t s) {
    const int cols = TcGeo<NP>::TCOLS;
    const int grid = (d.Pp / kTM) * d.C;
    const WalkSeg* none = nullptr;
    return pre ? launch_tc(k_walk_tc<NP, KC, true, false>, grid, tc_smem(cols), d.C, cols, s, ops, nops,
                           d.S, d.Sg, d.C, (double*)nullptr, ls, none, 0)
               : launch_tc(k_walk_tc<NP, KC, false, false>, grid, tc_smem(cols), d.C, cols, s, ops,
                           nops, d.S, d.Sg, d.C, cum, ls, none, 0);
}

template <int NP, int KC>
cudaError_t run_walk_tc_batch(const WalkSeg* segs, int nseg, int ntiles, bool pre,
                              const Dims& d, cudaStream_t s) {
    const int cols = TcGeo<NP>::TCOLS;
    const OpDesc* no_ops = nullptr;
    return pre ? launch_tc(k_walk_tc<NP, KC, true, true>, ntiles * d.C, tc_smem(cols), d.C, cols, s,
                           no_ops, 0, d.S, d.Sg, d.C, (double*)nullptr, 0, segs, nseg)
               : launch_tc(k_walk_tc<NP, KC, false, true>, ntiles * d.C, tc_smem(cols), d.C, cols, s,
                           no_ops, 0, d.S, d.Sg, d.C, (double*)nullptr, 0, segs, nseg);
}

template <int NP, int KC>
cudaError_t run_deriv_tc(const DerivDesc* desc, int nb, const double* catw, const double* patw,
                         const Dims& d, double* site, double* block, cudaStream_t s) {
    const int cols = TcGeo<NP>::DCOLS;
    const int ntiles = d.Pp / kTM;
    const DerivSeg* none = nullptr;
    return launch_tc(k_deriv_tc<NP, KC, false>, ntiles * d.C * nb, tc_smem(cols), d.C, cols, s, desc,
                     catw, patw, d.S, d.Sg, d.C, d.P, ntiles, site, block, none, 0);
}

template <int NP, int KC>
cudaError_t run_deriv_tc_batch(const DerivSeg* segs, int nseg, int nclusters, const Dims& d,
                               cudaStream_t s) {
    const int cols = TcGeo<NP>::DCOLS;
    const DerivDesc* no_desc = nullptr;
    const double* no_w = nullptr;
    return launch_tc(k_deriv_tc<NP, KC, true>, nclusters * d.C, tc_smem(cols), d.C, cols, s, no_desc,
                     no_w, no_w, d.S, d.Sg, d.C, 0, 1, (double*)nullptr, (double*)nullptr, segs,
                     nseg);
}

template <int NP, int KC>
cudaError_t run_prederiv_tc(const OpDesc* ops, const DerivDesc* dds, int nops, int nsum,
                            const double* catw, const double* patw, const Dims& d, int ls,
                            double* block, cudaStream_t s) {
    const int cols = TcFusedGeo<NP>::COLS;
    const size_t need = sizeof(TcFusedSmem) + 1024;
    const size_t floor_smem = tc_smem(cols);
    const size_t smem = need > floor_smem ? need : floor_smem;
    const int grid = (d.Pp / kTM) * d.C;
    const PreDerivSeg* none = nullptr;
    return launch_tc(k_prederiv_tc<NP, KC, false>, grid, smem, d.C, cols, s, ops, dds, nops, nsum,
                     d.S, d.Sg, d.C, d.P, catw, patw, ls, block, none, 0);
}

template <int NP, int KC>
cudaError_t run_prederiv_tc_batch(const PreDerivSeg* segs, int nseg, int ntiles, const Dims& d,
                                  cudaStream_t s) {
    const int cols = TcFusedGeo<NP>::COLS;
    const size_t need = sizeof(TcFusedSmem) + 1024;
    const size_t floor_smem = tc_smem(cols);
    const size_t smem = need > floor_smem ? need : floor_smem;
    const OpDesc* no_ops = nullptr;
    const DerivDesc* no_dds = nullptr;
    const double* no_w = nullptr;
    return launch_tc(k_prederiv_tc<NP, KC, true>, ntiles * d.C, smem, d.C, cols, s, no_ops, no_dds,
                     0, 0, d.S, d.Sg, d.C, 0, no_w, no_w, 0, (double*)nullptr, segs, nseg);
}

// (N, KC) of a padded state count: N = Sg rounded up to 16, KC as above.
#define B200_TC_DISPATCH(Sg, CALL)                                         \
    ((Sg) <= 8    ? CALL(16, 8)                                            \
     : (Sg) <= 16 ? CALL(16, 16)                                           \
     : (Sg) <= 32 ? CALL(32, 32)                                           \
     : (Sg) <= 48 ? CALL(48, 32)                                           \
                  : CALL(64, 32))

}  // namespace

bool tc_supported(const Dims& d) {
    return d.S > 4 && d.Sg <= 64 && d.C >= 1 && d.C <= 8 && d.Pp % kTM == 0;
}

int tc_tile_patterns() { return kTM; }

cudaError_t launch_opwalk_tc(const OpDesc* ops, int nops, bool pre, const Dims& d, double* cum,
                             int ls, cudaStream_t s) {
    if (nops == 0) return cudaSuccess;
    if (!tc_supported(d)) return cudaErrorInvalidValue;
#define WALK_(NP, KC) run_walk_tc<NP, KC>(ops, nops, pre, d, cum, ls, s)
    return B200_TC_DISPATCH(d.Sg, WALK_);
#undef WALK_
}

cudaError_t launch_deriv_tc(const DerivDesc* desc, int nb, const double* catw,
                            const double* patw, const Dims& d, double* site, double* block,
                            cudaStream_t s) {
    if (nb == 0) return cudaSuccess;
    if (!tc_supported(d)) return cudaErrorInvalidValue;
#define DER_(NP, KC) run_deriv_tc<NP, KC>(desc, nb, catw, patw, d, site, block, s)
    return B200_TC_DISPATCH(d.Sg, DER_);
#undef DER_
}

int prederiv_tc_blocks(const Dims& d) { return d.Pp / kTM; }

cudaError_t launch_prederiv_tc(const OpDesc* d_ops, const DerivDesc* d_desc, int nops, int nsum,
                               const double* catw, const double* patw, const Dims& d, int ls,
                               double* d_block, cudaStream_t s) {
    if (nops == 0) return cudaSuccess;
    if (!tc_supported(d)) return cudaErrorInvalidValue;
#define PD_(NP, KC) run_prederiv_tc<NP, KC>(d_ops, d_desc, nops, nsum, catw, patw, d, ls, d_block, s)
    return B200_TC_DISPATCH(d.Sg, PD_);
#undef PD_
}

cudaError_t launch_prederiv_tc_pairs(const OpDesc* d_ops, const DerivDesc* d_desc, int nops,
                                     int nsum, const double* catw, const double* patw,
                                     const Dims& d, int ls, double* d_block, cudaStream_t s) {
    if (nops == 0) return cudaSuccess;
    if (!tc_supported(d) || d.Sg <= 16 || d.Sg > 32 || nops % 2) return cudaErrorInvalidValue;
    const size_t need = sizeof(TcPairSmem) + 1024;
    const size_t floor_smem = tc_smem(kPairCols);
    const size_t smem = need > floor_smem ? need : floor_smem;
    const int grid = (d.Pp / kTM) * d.C;
    const PreDerivSeg* none = nullptr;
    return launch_tc(k_prederiv_tc_pairs<false>, grid, smem, d.C, kPairCols, s, d_ops, d_desc,
                     nops, nsum, d.S, d.Sg, d.C, d.P, catw, patw, ls, d_block, none, 0);
}

cudaError_t launch_prederiv_tc_pairs_batch(const PreDerivSeg* d_segs, int nseg, int ntiles,
                                           const Dims& d, cudaStream_t s) {
    if (nseg == 0 || ntiles == 0) return cudaSuccess;
    if (!tc_supported(d) || d.Sg <= 16 || d.Sg > 32) return cudaErrorInvalidValue;
    const size_t need = sizeof(TcPairSmem) + 1024;
    const size_t floor_smem = tc_smem(kPairCols);
    const size_t smem = need > floor_smem ? need : floor_smem;
    const OpDesc* no_ops = nullptr;
    const DerivDesc* no_dds = nullptr;
    const double* no_w = nullptr;
    return launch_tc(k_prederiv_tc_pairs<true>, ntiles * d.C, smem, d.C, kPairCols, s, no_ops,
                     no_dds, 0, 0, d.S, d.Sg, d.C, 0, no_w, no_w, 0, (double*)nullptr, d_segs,
                     nseg);
}

cudaError_t launch_prederiv_tc_batch(const PreDerivSeg* d_segs, int nseg, int ntiles,
                                     const Dims& d, cudaStream_t s) {
    if (nseg == 0 || ntiles == 0) return cudaSuccess;
    if (!tc_supported(d)) return cudaErrorInvalidValue;
#define PDB_(NP, KC) run_prederiv_tc_batch<NP, KC>(d_segs, nseg, ntiles, d, s)
    return B200_TC_DISPATCH(d.Sg, PDB_);
#undef PDB_
}

// Whether the tensor-core derivative kernel of this shape can launch without
// oversubscribing TMEM (the check launch_tc makes before launching).
template <int NP, int KC>
bool deriv_tc_fits() {
    const int cols = TcGeo<NP>::DCOLS;
    const size_t smem = tc_smem(cols);
    if (cudaFuncSetAttribute(k_deriv_tc<NP, KC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_deriv_tc<NP, KC, true>, kTT, smem) !=
        cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return per_sm * cols <= 512;
}

bool deriv_tc_launchable(const Dims& d) {
    if (!tc_supported(d)) return false;
#define FIT_(NP, KC) deriv_tc_fits<NP, KC>()
    return B200_TC_DISPATCH(d.Sg, FIT_);
#undef FIT_
}

cudaError_t launch_walk_tc_batch(const WalkSeg* d_segs, int nseg, int ntiles, bool pre,
                                const Dims& d, cudaStream_t s) {
    if (nseg == 0 || ntiles == 0) return cudaSuccess;
    if (!tc_supported(d)) return cudaErrorInvalidValue;
#define WALKB_(NP, KC) run_walk_tc_batch<NP, KC>(d_segs, nseg, ntiles, pre, d, s)
    return B200_TC_DISPATCH(d.Sg, WALKB_);
#undef WALKB_
}

cudaError_t launch_deriv_tc_batch(const DerivSeg* d_segs, int nseg, int nclusters, const Dims& d,
                                  cudaStream_t s) {
    if (nseg == 0 || nclusters == 0) return cudaSuccess;
    if (!tc_supported(d)) return cudaErrorInvalidValue;
#define DERB_(NP, KC) run_deriv_tc_batch<NP, KC>(d_segs, nseg, nclusters, d, s)
    return B200_TC_DISPATCH(d.Sg, DERB_);
#undef DERB_
}

// ------------------------------------------------------- TMA tensor maps
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).  Partials [Pp][C][Sg] (FP32): a 3-D map
// {Sg, C, Pp} with box {KC, 1, 128}; matrices [C][Sg][Sg]: {Sg, Sg, C} with
// box {KC, NP, 1}.  Elements past Sg are zero-filled; with KC = 32 (128-byte
// rows) the 128-byte swizzle, otherwise none.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        (void)cudaGetLastError();
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

static int tc_np(int Sg) { return Sg <= 16 ? 16 : Sg <= 32 ? 32 : Sg <= 48 ? 48 : 64; }

cudaError_t tc_encode_map(TmaMap* out, const void* base, bool matrix, const Dims& d) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn || !tc_supported(d)) return cudaErrorNotSupported;
    const int NP = tc_np(d.Sg), KC = kTK;
    cuuint64_t dims[3], strides[2];
    cuuint32_t box[3], es[3] = {1, 1, 1};
    if (!matrix) {
        dims[0] = (cuuint64_t)d.Sg; dims[1] = (cuuint64_t)d.C; dims[2] = (cuuint64_t)d.Pp;
        strides[0] = (cuuint64_t)d.Sg * 4; strides[1] = (cuuint64_t)d.C * d.Sg * 4;
        box[0] = (cuuint32_t)KC; box[1] = 1; box[2] = (cuuint32_t)kTM;
    } else {
        dims[0] = (cuuint64_t)d.Sg; dims[1] = (cuuint64_t)d.Sg; dims[2] = (cuuint64_t)d.C;
        strides[0] = (cuuint64_t)d.Sg * 4; strides[1] = (cuuint64_t)d.Sg * d.Sg * 4;
        box[0] = (cuuint32_t)KC; box[1] = (cuuint32_t)NP; box[2] = 1;
    }
    const CUresult r = fn(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                          const_cast<void*>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int NP>
cudaError_t run_walk_tc_tma(const OpDesc* ops, const TcOpMaps* maps, int nops, bool pre,
                            const Dims& d, double* cum, int ls, cudaStream_t s) {
    const int cols = TcGeo<NP>::TCOLS;
    const int grid = (d.Pp / kTM) * d.C;
    const size_t need = sizeof(TcTma) + 1024;
    const size_t floor_smem = tc_smem(cols);
    const size_t smem = need > floor_smem ? need : floor_smem;
    return pre ? launch_tc(k_walk_tc_tma<NP, true>, grid, smem, d.C, cols, s, ops, maps, nops,
                           d.S, d.Sg, d.C, (double*)nullptr, ls)
               : launch_tc(k_walk_tc_tma<NP, false>, grid, smem, d.C, cols, s, ops, maps, nops,
                           d.S, d.Sg, d.C, cum, ls);
}

cudaError_t launch_opwalk_tc_tma(const OpDesc* ops, const TcOpMaps* maps, int nops, bool pre,
                                 const Dims& d, double* cum, int ls, cudaStream_t s) {
    if (nops == 0) return cudaSuccess;
    if (!tc_supported(d) || !encode_tiled()) return cudaErrorInvalidValue;
    switch (tc_np(d.Sg)) {
        case 16: return run_walk_tc_tma<16>(ops, maps, nops, pre, d, cum, ls, s);
        case 32: return run_walk_tc_tma<32>(ops, maps, nops, pre, d, cum, ls, s);
        case 48: return run_walk_tc_tma<48>(ops, maps, nops, pre, d, cum, ls, s);
        default: return run_walk_tc_tma<64>(ops, maps, nops, pre, d, cum, ls, s);
    }
}

cudaError_t tc_status_async(int* pinned_dst, cudaStream_t s) {
    return cudaMemcpyFromSymbolAsync(pinned_dst, b200_tc_status, sizeof(int), 0,
                                     cudaMemcpyDeviceToHost, s);
}

cudaError_t tc_raise_status(cudaStream_t s) {
    static const int one = 1;
    return cudaMemcpyToSymbolAsync(b200_tc_status, &one, sizeof(int), 0,
                                   cudaMemcpyHostToDevice, s);
}

cudaError_t tc_clear_status(cudaStream_t s) {
    static const int zero = 0;
    cudaError_t e = cudaMemcpyToSymbolAsync(b200_tc_status, &zero, sizeof(int), 0,
                                            cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

}  // namespace b200
