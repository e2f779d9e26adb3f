// Host-callable launchers of the sm_100a kernels.  Every launcher takes device
// pointers, sizes and the instance's stream and returns a cudaError_t; none of
// them allocates.
#pragma once
#include <cuda_runtime.h>
#include "b200_types.h"

namespace b200 {

struct Dims {
    int S;       // states
    int Sg;      // padded state stride
    int P;       // patterns (unpadded)
    int Pp;      // padded patterns
    int C;       // rate categories
};

// Transition matrices from the eigen cube (FP64), stored as Real.
template <typename Real>
cudaError_t launch_update_matrices(const MatJob* d_jobs, int njobs, const Dims& d,
                                   cudaStream_t s);
// result[m] = A[m] . B[m] per category (convolution), or transpose A.
template <typename Real>
cudaError_t launch_matrix_pairs(const void* const* d_a, const void* const* d_b,
                                void* const* d_out, int n, int op, const Dims& d,
                                cudaStream_t s);

// Post-order partials over an op list (S = 4), one launch for the whole list.
// `variant` selects the kernel shape (see s4_walk_variants; < 0 = default).
// `ranged`: some op has its own pattern range or cumulative buffer (partition
// ops); without it the lane-group kernels skip those per-op checks.
// `h_ops`, when given, is the host copy of the list (for the variants that
// take it as a kernel parameter).
template <typename Real>
cudaError_t launch_update_partials(const OpDesc* d_ops, int nops, const Dims& d,
                                   double* cumulative, int log_scalers, cudaStream_t s,
                                   int variant = -1, bool ranged = true,
                                   const OpDesc* h_ops = nullptr);
// Pre-order partials over an op list (S = 4).
template <typename Real>
cudaError_t launch_update_pre_partials(const OpDesc* d_ops, int nops, const Dims& d,
                                       int log_scalers, cudaStream_t s, int variant = -1,
                                       bool ranged = true, const OpDesc* h_ops = nullptr);
// Number of S = 4 op-walk variants for C categories (variants 0 .. n-1).
int s4_walk_variants(int C);

// The same op lists for S != 4 (S <= 64, C <= 8): clustered CUDA-core kernels.
// dep[o] != 0 when op o reads the output of op o - 1.
template <typename Real>
cudaError_t launch_opwalk_generic(const OpDesc* d_ops, const uint8_t* d_dep, int nops, bool pre,
                                  const Dims& d, double* cumulative, int log_scalers,
                                  cudaStream_t s);
template <typename Real>
cudaError_t launch_deriv_generic(const DerivDesc* d_desc, int nb, const double* catw,
                                 const double* patw, const Dims& d, double* d_site,
                                 double* d_block, cudaStream_t s);
// Pattern tile of the clustered kernels (one derivative partial per tile).
int generic_tile_patterns(int Sg, bool dbl);

// The FP32 op lists and edge derivatives for 4 < S <= 64 on the tensor cores
// (tcgen05, 3 x tf32 split products), k_tc.cu.  Same arguments and results as
// the clustered CUDA-core kernels; one derivative partial per tc_tile_patterns()
// patterns.  A launch that cannot guarantee TMEM for every resident CTA is
// refused with cudaErrorInvalidConfiguration.
bool tc_supported(const Dims& d);
int tc_tile_patterns();
cudaError_t launch_opwalk_tc(const OpDesc* d_ops, int nops, bool pre, const Dims& d,
                             double* cumulative, int log_scalers, cudaStream_t s);
cudaError_t launch_deriv_tc(const DerivDesc* d_desc, int nb, const double* catw,
                            const double* patw, const Dims& d, double* d_site, double* d_block,
                            cudaStream_t s);
// Batched tensor-core walks and derivatives over instances with one (S, C),
// FP32 (d gives S, Sg and C; its pattern counts are unused).  Walk segments
// count pattern tiles of 128 in first_cta; derivative segments count
// (branch, tile) clusters, nblk = the instance's tiles.
cudaError_t launch_walk_tc_batch(const WalkSeg* d_segs, int nseg, int ntiles, bool pre,
                                 const Dims& d, cudaStream_t s);
cudaError_t launch_deriv_tc_batch(const DerivSeg* d_segs, int nseg, int nclusters, const Dims& d,
                                  cudaStream_t s);
bool deriv_tc_launchable(const Dims& d);
// Fused pre-order walk + edge derivatives on the tensor cores (FP32, S > 4):
// ops as launch_opwalk_tc's pre-order list, d_desc[k] the derivative of op k's
// branch (post = the node's post-order operand, pre = op k's destination);
// the sums of op k into d_block rows k and nsum + k, prederiv_tc_blocks(d)
// partials each (add them with launch_final_sum).
int prederiv_tc_blocks(const Dims& d);
// ... over several instances with one (S, C): segment first_cta counts
// 128-pattern tiles, ntiles their total; each segment's sums into its block.
cudaError_t launch_prederiv_tc_batch(const PreDerivSeg* d_segs, int nseg, int ntiles,
                                     const Dims& d, cudaStream_t s);
cudaError_t launch_prederiv_tc(const OpDesc* d_ops, const DerivDesc* d_desc, int nops, int nsum,
                               const double* catw, const double* patw, const Dims& d, int ls,
                               double* d_block, cudaStream_t s);
// The same for 17 to 32 padded states on lists made only of sibling pairs
// (OpDesc::kind kPairFirst on every even op; the caller checks): a pair a
// step, each post-order tile feeding two products (k_prederiv_tc_pairs).
// cudaErrorInvalidValue for other shapes.
cudaError_t launch_prederiv_tc_pairs(const OpDesc* d_ops, const DerivDesc* d_desc, int nops,
                                     int nsum, const double* catw, const double* patw,
                                     const Dims& d, int ls, double* d_block, cudaStream_t s);
// Its batched form over segments as launch_prederiv_tc_batch (every
// segment's list made of sibling pairs; the caller checks).
cudaError_t launch_prederiv_tc_pairs_batch(const PreDerivSeg* d_segs, int nseg, int ntiles,
                                           const Dims& d, cudaStream_t s);
// TMA-fed tensor-core walk (FP32, 4 < S <= 64): maps[k] gives op k's tensor
// maps (tc_encode_map: a partials buffer, or a matrix buffer, of this shape).
cudaError_t tc_encode_map(TmaMap* out, const void* base, bool matrix, const Dims& d);
cudaError_t launch_opwalk_tc_tma(const OpDesc* d_ops, const TcOpMaps* d_maps, int nops, bool pre,
                                 const Dims& d, double* cum, int ls, cudaStream_t s);
// The flag a tensor-core kernel sets when a bounded wait on its tensor-core
// work timed out: queue its copy into pinned host memory on `s` (read it after
// the stream completes), and clear it (synchronises `s`).
cudaError_t tc_status_async(int* pinned_dst, cudaStream_t s);
cudaError_t tc_clear_status(cudaStream_t s);
cudaError_t tc_raise_status(cudaStream_t s);      // as a timed-out wait would
// The same for the bulk-copy derivative stream (k_reduce.cu); clearing does
// not synchronise.
cudaError_t bulk_status_async(int* pinned_dst, cudaStream_t s);
cudaError_t bulk_clear_status(cudaStream_t s);
cudaError_t bulk_raise_status(cudaStream_t s);    // as a timed-out wait would

// Root log-likelihood: site lnL into d_site[P]; the weighted total into d_out[0].
// d_block holds root_blocks(d, P, wide) doubles: `wide` spreads a pattern
// over several lanes (root_lanes), otherwise one thread per pattern and
// reduction_blocks(P) partial sums.
template <typename Real>
cudaError_t launch_root_lnl(const void* root, const double* catw, const double* freqs,
                            const double* cumulative, const double* patw, const Dims& d,
                            double* d_site, double* d_block, double* d_out, cudaStream_t s,
                            bool wide = true);
// The same over patterns [p_begin, p_end) (one partition); d_block holds
// root_blocks(d, p_end - p_begin, wide) doubles.
template <typename Real>
cudaError_t launch_root_lnl_range(const void* root, const double* catw, const double* freqs,
                                  const double* cumulative, const double* patw, const Dims& d,
                                  int p_begin, int p_end, double* d_site, double* d_block,
                                  double* d_out, cudaStream_t s, bool wide = true);
int root_lanes(const Dims& d);
int root_blocks(const Dims& d, int n, bool wide);

// Edge log-likelihood (+ optional first / second derivative sums).
template <typename Real>
cudaError_t launch_edge_lnl(const void* parent, const void* child, int child_is_states,
                            const void* pmat, double ppad, const void* d1mat, double d1pad,
                            const void* d2mat, double d2pad, const double* catw,
                            const double* freqs, const double* cumulative,
                            const double* patw, const Dims& d, double* d_site,
                            double* d_site1, double* d_site2, double* d_block,
                            double* d_out, cudaStream_t s);

// The same over patterns [p_begin, p_end) only: d_out gets that range's three
// sums, d_site / d_site1 / d_site2 only its entries.
template <typename Real>
cudaError_t launch_edge_lnl_range(const void* parent, const void* child, int child_is_states,
                                  const void* pmat, double ppad, const void* d1mat, double d1pad,
                                  const void* d2mat, double d2pad, const double* catw,
                                  const double* freqs, const double* cumulative,
                                  const double* patw, const Dims& d, int p_begin, int p_end,
                                  double* d_site, double* d_site1, double* d_site2,
                                  double* d_block, double* d_out, cudaStream_t s);

// Edge derivatives for `nb` branches; per-site values optional (d_site may be
// null), sums and sums of squares into d_sums[2*nb].  d_block holds
// 2 * nb * deriv_blocks(d) doubles of per-block partial sums.  `variant`
// selects the S = 4 kernel shape (0 .. deriv4_variants(d) - 1; < 0 = default).
template <typename Real>
cudaError_t launch_edge_derivatives(const DerivDesc* d_desc, int nb, const double* catw,
                                    const double* patw, const Dims& d, double* d_site,
                                    double* d_block, double* d_sums, cudaStream_t s,
                                    int variant = -1);
int deriv4_variants(const Dims& d);

// cumulative[p] += sign * sum_i f(scale[idx_i][p]), f = identity (log scalers) or log.
cudaError_t launch_accumulate_scale(double* cumulative, const double* pool, const int* d_idx,
                                    int n, int Pp, int P, double sign, int log_scalers,
                                    int p_begin, int p_end, cudaStream_t s);

// Fill a partials buffer with the state frequencies (pre-order root).
template <typename Real>
cudaError_t launch_fill_root(void* dest, const double* freqs, const Dims& d, cudaStream_t s);

// Number of per-block partial sums used by the reductions above.
int reduction_blocks(int Pp);
// ... and by one branch of an edge-derivative launch (S = 4 kernels).
int deriv_blocks(const Dims& d);
// Final pass of an edge-derivative launch: sums[k] over nblk block partials.
cudaError_t launch_deriv_final(const double* d_block, int nblk, int nb, double* d_sums,
                               cudaStream_t s);
// out[k] = the fixed-order sum of block[k * nblk .. k * nblk + nblk), k < nout.
cudaError_t launch_final_sum(const double* d_block, int nblk, int nout, double* d_out,
                             cudaStream_t s);
// Post-order walk + scale accumulation + root lnL in one launch (S = 4, C in
// {1, 2, 4, 8}, at most 256 ops, the root the last op's destination; k_partials.cu):
// the list's scale buffers as updatePartials writes them; with `cum`, its
// patterns' sums of log scale factors (reset, then accumulated); site lnL into
// `site`, the weighted total into out[0].  `block` holds post_root_blocks(d)
// doubles.
// The same over many 4-state instances (segments as k_walk4_batch; one
// launch per category count, ncta = the segments' total CTAs, each CTA
// post_root_batch_patterns(C) patterns; every member's block partials are
// post_root_blocks of its shape).
int post_root_batch_patterns(int C);
template <typename Real>
cudaError_t launch_post4_root_batch(const PostRootSeg* d_segs, int nseg, int ncta, int C,
                                    cudaStream_t s);
int post_root_blocks(const Dims& d);
template <typename Real>
cudaError_t launch_post4_root(const OpDesc* h_ops, int nops, const Dims& d, double* cum, int ls,
                              const double* catw, const double* freqs, const double* patw,
                              double* site, double* block, double* out, cudaStream_t s);
// The same with the sums to d_sums[0, nb) and the sums of squares to
// d_sumsq[0, nb) (a slice of a longer list's output).
cudaError_t launch_deriv_final_at(const double* d_block, int nblk, int nb, double* d_sums,
                                  double* d_sumsq, cudaStream_t s);

// Fused pre-order partials + edge derivatives (k_fused.cu): S = 4, C in
// {1, 2, 4, 8}, any list length (one launch per 256 ops).  d_block needs
// 2 * nops * fused_blocks(d) doubles; d_sums receives the nops sums, then the
// nops sums of squares.
// Cross-product derivative sums (k_reduce.cu), S <= 64: d_out receives the
// S * S sums over the nb branches (desc: post, pre, post_is_states used; fac
// [nb][C] = w_c r_c t_b); d_block needs S * S * ceil(P / cross_tile_patterns)
// doubles.
int cross_tile_patterns(const Dims& d, bool dbl);
template <typename Real>
cudaError_t launch_cross_products(const DerivDesc* d_desc, int nb, const double* catw,
                                  const double* fac, const double* patw, const Dims& d,
                                  double* d_block, double* d_out, cudaStream_t s);

bool fused_supported(const Dims& d, int nops);
int fused_blocks(const Dims& d);
// variant 1: the walk of k_fused.cu; 2: pairs-only FP32 lists, 2 patterns a
// thread (cudaErrorInvalidValue for other lists).
template <typename Real>
cudaError_t launch_pre_deriv4(const PreDerivOp* h_ops, int nops, const Dims& d,
                              const double* catw, const double* patw, int ls, double* d_block,
                              double* d_sums, cudaStream_t s, int variant);

// Batched fused pre-order walk + edge derivatives (S = 4, C in {1, 2, 4, 8};
// k_fused.cu): one CTA per pre_deriv4_batch_patterns(C) patterns of a member;
// a member's sums of op k into its block rows k and nops + k, nblk = its CTAs
// x 8 warp partials each.
int pre_deriv4_batch_patterns(int C);
template <typename Real>
cudaError_t launch_pre_deriv4_batch(const PreDerivSeg* d_segs, int nseg, int ncta, int C,
                                    cudaStream_t s);

// ---- batched launches over several instances (segment tables on the device;
// ncta = the segments' total CTAs; see b200_types.h) ------------------------
// S = 4 walks, one pattern per thread (256-thread CTAs of 256 / C patterns);
// C in {1, 2, 4, 8}.
template <typename Real>
cudaError_t launch_walk4_batch(const WalkSeg* d_segs, int nseg, int ncta, int C, bool pre,
                               cudaStream_t s);
// S = 4 edge derivatives (one CTA per deriv4_batch_tile(C) patterns of a branch).
int deriv4_batch_tile(int C);
template <typename Real>
cudaError_t launch_deriv4_batch(const DerivSeg* d_segs, int nseg, int ncta, int C,
                                cudaStream_t s);
// Root log-likelihoods (one CTA per reduction_blocks' 128 patterns).
template <typename Real>
cudaError_t launch_root_batch(const RootSeg* d_segs, int nseg, int ncta, cudaStream_t s);
// Scale-factor accumulation (one CTA per accumulate_batch_patterns() patterns).
int accumulate_batch_patterns();
cudaError_t launch_accumulate_batch(const AccSeg* d_segs, int nseg, int ncta, cudaStream_t s);
// Final sums of block partials: one CTA per output (nout in total).
cudaError_t launch_final_batch(const FinalSeg* d_segs, int nseg, int nout, cudaStream_t s);
// Pre-order root fills (one CTA per 256 values).
template <typename Real>
cudaError_t launch_fill_batch(const FillSeg* d_segs, int nseg, int ncta, cudaStream_t s);

}  // namespace b200

