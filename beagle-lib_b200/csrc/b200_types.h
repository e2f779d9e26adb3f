// Types shared by the host instance (b200_instance.cpp) and the sm_100a
// kernels (k_*.cu).  Plain C++: no CUDA qualifiers, so g++ and nvcc agree on
// the layout.
#pragma once
#include <cstdint>

namespace b200 {

// Device-side layout of one instance (all buffers are in this GPU's HBM):
//   partials   [pattern Pp][category C][state Sg]   Real   (pattern-major)
//   tip states [pattern Pp]                          int32  (S = missing state)
//   matrices   [category C][row Sg][col Sg]          Real   (zero padded)
//   scale      [pattern Pp]                          double
// Sg = S rounded up to a multiple of 4 (one 16-byte row per pattern for S = 4),
// Pp = P rounded up to a multiple of kPatternPad so pattern tiles need no tail.
// Every matrix also has a transposed image (same layout, P^T), kept in step by
// whatever writes the matrix, so kernels stage either orientation by a plain
// contiguous copy.
constexpr int kPatternPad = 128;

enum OpKind : int {
    kX1States = 1,      // first operand is a compact tip-state buffer
    kX2States = 2,      // second operand is a compact tip-state buffer
    kM1Transposed = 4,  // pre-order: the node's matrix is given as its transpose
    kPostStates = 8,    // fused pre-order op: the node's own post-order operand is tip states
    kPairFirst = 16,    // fused pre-order op: this op and the next are a sibling pair
    kPairMats = 32,     // ... whose two ops use the same two matrices, untransposed
    kPairD = 64,        // ... whose two branches share one derivative matrix
};

// One resolved partials operation (post-order or pre-order).  Post-order:
// dest = (M1 . x1) * (M2 . x2).  Pre-order: x1 = parent pre-partials, x2 =
// sibling post-partials, dest[j] = sum_i M1[i][j] * x1[i] * (M2 . x2)[i].
struct OpDesc {
    const void* x1;
    const void* x2;
    void* dest;
    const void* m1;
    const void* m2;
    const void* m1t;            // transposed images of m1 / m2 ([C][Sg][Sg], P^T)
    const void* m2t;
    double* scale_write;        // rescale into this buffer (nullptr = no rescale)
    const double* scale_read;   // divide by these stored factors (nullptr = none)
    double pad1;                // value of the missing-state column of M1
    double pad2;                // ... of M2
    double* cum;                // cumulative scale buffer of this op (partition ops) or null
    int kind;                   // OpKind bits
    int p_begin;                // only patterns [p_begin, p_end) are written: the op's
    int p_end;                  //   partition, or [0, Pp) for a whole-instance op
    int slots;                  // shared-memory slots of the S = 4 slot walks (kSlot*)
};

// OpDesc::slots packs three 4-bit fields, each a slot index + 1 (0 = none):
// the slot that keeps the op's result for a later op of the same list (bits
// 0-3), and the slots its operands x1 (bits 4-7) and x2 (bits 8-11) are read
// from instead of device memory.  Only whole-instance lists get slots.
constexpr int kMaxSlots = 8;
#ifdef __CUDACC__
__host__ __device__
#endif
inline int slot_field(int packed, int field) { return ((packed >> (4 * field)) & 15) - 1; }

// One op of the fused pre-order + edge-derivative walk (S = 4): the
// pre-order op (dest = P_node^T (parent o P_sib sib)) and the derivative of the
// node's branch from its new pre-order row and its post-order operand.
struct PreDerivOp {
    const void* parent;         // parent's pre-order partials
    const void* sib;            // sibling's post-order partials or tip states
    void* dest;                 // this node's pre-order partials
    const void* mnode;          // P of this node's branch (transposed if kM1Transposed)
    const void* msib;           // P of the sibling's branch
    const void* post;           // this node's post-order partials or tip states
    const void* dmat;           // derivative matrix of this node's branch
    double* scale_write;        // rescale into this buffer (nullptr = none)
    double pad_sib;             // missing-state value of msib
    double dpad;                // missing-state value of dmat
    int kind;                   // OpKind bits: kX2States, kM1Transposed, kPostStates, kPairFirst
    int reserved;
};

// An opaque TMA tensor map (CUtensorMap: 128 bytes, 64-byte aligned) in
// device memory, and the four maps one tensor-core op reads through: the
// partials of its two operands and their matrices (null: not a partials
// operand).
struct alignas(64) TmaMap {
    unsigned char bytes[128];
};
struct TcOpMaps {
    const TmaMap* a1;
    const TmaMap* a2;
    const TmaMap* b1;
    const TmaMap* b2;
};

// One branch of an edge-derivative launch.
struct DerivDesc {
    const void* post;           // post-order partials (or tip states) below the branch
    const void* pre;            // pre-order partials of the same node
    const void* dmat;           // derivative matrix [C][Sg][Sg]
    const void* dmatt;          // its transposed image
    double dpad;                // its missing-state column value
    int post_is_states;
    int reserved;
};

// One matrix of a transition-matrix launch: P (and optionally dP/dt, d2P/dt2)
// for branch length t under category rates `rates`.
struct MatJob {
    void* p;
    void* d1;
    void* d2;
    void* pt;                   // transposed images (written alongside)
    void* d1t;
    void* d2t;
    const double* cube;         // eigen cube [S][S][S] (i, k, j)
    const double* evals;        // eigenvalues [S]
    const double* rates;        // category rates [C]
    double t;
    // Model categories: category c uses eigen system cat_eig[c] (cube and
    // evals are then the bases of all systems) with rate 1; null otherwise.
    const int* cat_eig;
    // Branch length read on the device at run time instead of `t` (a CUDA
    // graph's lengths buffer); null otherwise.
    const double* tlen;
};

// ---- batched launches over several instances (b200_batch.cpp) ----------
// Each launch takes one segment per instance; a CTA finds its segment by
// binary search over the segments' first_cta (ascending, first one 0).

// One instance's op list in a batched S = 4 walk (one pattern per thread).
struct WalkSeg {
    const OpDesc* ops;
    double* cum;                // cumulative scale buffer of a post-order list, or null
    int nops;
    int Pp;
    int log_scalers;
    int first_cta;
};

// One instance's branches in a batched S = 4 edge-derivative launch.
struct DerivSeg {
    const DerivDesc* desc;
    const double* catw;
    const double* patw;
    double* block;              // this instance's 2 * nb * nblk block partial sums
    int nb;
    int P;
    int nblk;                   // blocks per branch
    int first_cta;
};

// One instance's list in a batched fused pre-order + edge-derivative launch.
struct PreDerivSeg {
    const PreDerivOp* fops;     // S = 4: the fused op list
    const OpDesc* ops;          // S > 4 (tensor cores): the pre-order walk table
    const DerivDesc* dds;       //   ... and the derivative of each op's branch
    const double* catw;
    const double* patw;
    double* block;              // this instance's 2 * nops * nblk block partial sums
    int nops;
    int P;
    int Pp;
    int nblk;                   // block partials per output
    int log_scalers;
    int first_cta;              // S = 4: CTAs; tensor cores: 128-pattern tiles
};

// One instance's root log-likelihood in a batched launch (any state count).
struct RootSeg {
    const void* root;
    const double* catw;
    const double* freqs;
    const double* cum;          // or null
    const double* patw;
    double* site;               // site log-likelihoods [P]
    double* block;              // block partial sums [nblk]
    int S, Sg, C, P;
    int first_cta;
    int reserved;
};

// One instance's fused post-order walk with scale accumulation and root lnL
// in a batched launch (k_post4root_batch).
struct PostRootSeg {
    const OpDesc* ops;
    double* cum;                // cumulative scale buffer (written once), or null
    const double* catw;
    const double* freqs;
    const double* patw;
    double* site;               // site log-likelihoods [P]
    double* block;              // one partial sum per warp
    int nops;
    int Pp;
    int P;
    int log_scalers;
    int first_cta;
    int reserved;
};

// One instance's scale-factor accumulation (optionally after resetting the
// cumulative buffer) in a batched launch.
struct AccSeg {
    double* cum;
    const double* pool;         // the instance's scale buffers, Pp doubles each
    const int* idx;             // scale buffer indices to add
    int n;
    int Pp;
    int P;
    int log_scalers;
    int reset;
    int first_cta;
};

// One instance's pre-order root partials (state frequencies) in a batched fill.
struct FillSeg {
    void* dest;
    const double* freqs;
    long long n;                // Pp * C * Sg values
    int S, Sg;
    int first_cta;
    int reserved;
};

// Outputs [first_out, first_out + nout) of a batched final sum: out[k] = sum of
// the nblk block partials block[k * nblk ...].
struct FinalSeg {
    const double* block;
    double* out;
    int nblk;
    int nout;
    int first_out;
    int reserved;
};

}  // namespace b200

