// Host side of one B200 instance: the buffer registry, flag handling, op
// validation and kernel launches behind every beagleB200* call.  It mirrors
// the reference's BeagleImpl interface (libhmsbeagle/BeagleImpl.h:31-268):
// same method set, same argument meaning, same return codes.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "b200_kernels.h"

namespace b200 {

// A device buffer that only grows; used for per-call tables and scratch.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    std::vector<uint8_t> last;     // last uploaded contents (upload is skipped if equal)
    unsigned epoch = 0;            // graph-launch epoch of `last`
    cudaError_t reserve(size_t n);
    cudaError_t upload(const void* src, size_t n, cudaStream_t s);
    void release();
};

// Every CUDA-graph launch (of an instance or a batch) starts a new upload
// epoch: a graph's copy nodes rewrite tables behind DevBuf::last, so an
// upload skips only when nothing was launched since its previous copy.  While
// a thread captures, every upload copies (through graph-owned pinned memory).
void note_graph_launch();
// Graph-owned pinned blocks of the capture this thread is recording (null
// when not capturing).
std::vector<void*>*& capture_pinned();

class Instance {
public:
    ~Instance();

    // beagleCreateInstance (BeagleImpl.h:36-48); returns a BeagleReturnCode.
    int create(int tipCount, int partialsBufferCount, int compactBufferCount, int stateCount,
               int patternCount, int eigenBufferCount, int matrixBufferCount, int categoryCount,
               int scaleBufferCount, int device, long preferenceFlags, long requirementFlags);

    long flags() const { return flags_; }
    cudaStream_t stream() const { return stream_; }
    int device() const { return device_; }
    const char* implName() const { return dbl_ ? "B200-sm100a-Double" : "B200-sm100a-Mixed"; }

    int setTipStates(int tipIndex, const int* inStates);
    int setTipPartials(int tipIndex, const double* inPartials);
    int setPartials(int bufferIndex, const double* inPartials);
    int setRootPrePartials(const int* bufferIndices, const int* freqIndices, int count);
    int getPartials(int bufferIndex, int scaleIndex, double* outPartials);
    int setEigenDecomposition(int eigenIndex, const double* evec, const double* ivec,
                              const double* evals);
    int setStateFrequencies(int index, const double* freqs);
    int setCategoryWeights(int index, const double* weights);
    int setCategoryRates(const double* rates) { return setCategoryRatesWithIndex(0, rates); }
    int setCategoryRatesWithIndex(int index, const double* rates);
    int setPatternWeights(const double* weights);
    int setPatternPartitions(int partitionCount, const int* partitions);

    int setTransitionMatrix(int matrixIndex, const double* inMatrix, double paddedValue);
    int setTransitionMatrices(const int* matrixIndices, const double* inMatrices,
                              const double* paddedValues, int count);
    int getTransitionMatrix(int matrixIndex, double* outMatrix);
    int transposeTransitionMatrices(const int* in, const int* out, int count);
    int convolveTransitionMatrices(const int* first, const int* second, const int* result,
                                   int count);
    int updateTransitionMatrices(int eigenIndex, const int* probIdx, const int* d1Idx,
                                 const int* d2Idx, const double* edgeLengths, int count);
    int updateTransitionMatricesWithMultipleModels(const int* eigenIndices,
                                                   const int* rateIndices, const int* probIdx,
                                                   const int* d1Idx, const int* d2Idx,
                                                   const double* edgeLengths, int count);
    int updateTransitionMatricesWithModelCategories(const int* eigenIndices, const int* probIdx,
                                                    const int* d1Idx, const int* d2Idx,
                                                    const double* edgeLengths, int count);

    int updatePartials(const int* ops, int count, int cumulativeScaleIndex);
    int updatePrePartials(const int* ops, int count, int cumulativeScaleIndex);
    int updatePartialsByPartition(const int* ops, int count);
    int updatePrePartialsByPartition(const int* ops, int count);
    int waitForPartials();

    int accumulateScaleFactors(const int* idx, int count, int cumulative, double sign,
                               int partition);
    int resetScaleFactors(int cumulative, int partition);
    int copyScaleFactors(int dst, int src);
    int getScaleFactors(int src, double* out);

    int calculateRootLogLikelihoods(const int* bufs, const int* cw, const int* sf,
                                    const int* cum, int count, double* out);
    int calculateRootLogLikelihoodsByPartition(const int* bufs, const int* cw, const int* sf,
                                               const int* cum, const int* parts, int nparts,
                                               int count, double* outByPart, double* out);
    int calculateEdgeDerivatives(const int* post, const int* pre, const int* dmat,
                                 const int* cw, int count, double* outDerivs, double* outSum,
                                 double* outSumSq);
    // Kernel variant last run per autotuner kind (1 post-order walk, 2
    // pre-order walk, 3 edge derivatives, 4 fused pre-order + derivatives;
    // -1 = default shape, -2 = not run yet).
    int picked(int kind) const { return kind >= 1 && kind <= 4 ? picked_[kind] : -2; }
    int calculateCrossProducts(const int* post, const int* pre, const int* rates_idx,
                               const int* cw, const double* lengths, int count,
                               double* outSum);
    // updatePartials + (reset and accumulate of the list's scale factors) +
    // calculateRootLogLikelihoods in one walk (S = 4) or as those calls.
    int updatePartialsWithRootLogLikelihood(const int* ops, int count, int cumulative, int root,
                                            int cw, int sf, double* out);
    // updatePrePartials + calculateEdgeDerivatives (sums only) in one walk.
    int updatePrePartialsWithDerivatives(const int* ops, int count, const int* post,
                                         const int* dmat, const int* cw, double* outSum,
                                         double* outSumSq);
    int calculateEdgeLogLikelihoods(const int* parents, const int* children, const int* prob,
                                    const int* d1, const int* d2, const int* cw, const int* sf,
                                    const int* cum, int count, double* outLnL, double* outD1,
                                    double* outD2);
    int calculateEdgeLogLikelihoodsByPartition(const int* parents, const int* children,
                                               const int* prob, const int* d1, const int* d2,
                                               const int* cw, const int* sf, const int* cum,
                                               const int* parts, int nparts, int count,
                                               double* outByPart, double* out,
                                               double* outD1ByPart, double* outD1,
                                               double* outD2ByPart, double* outD2);
    int getLogLikelihood(double* out);
    int getDerivatives(double* d1, double* d2);
    int getSiteLogLikelihoods(double* out);
    int getSiteDerivatives(double* d1, double* d2);

    // CUDA graphs of an ASYNCH instance's work (beagleB200BeginCapture ...).
    int beginCapture();
    int endCapture(int* graph);
    int launchGraph(int graph);
    // Raise, on this instance's stream, the device flag a kernel sets when a
    // bounded wait runs out (which 0: tensor-core kernels, 1: bulk-copy
    // derivative), as if one had; the next result call reports it.
    int injectKernelTimeout(int which);
    int launchGraphWithLengths(int graph, const double* lengths, int count);

    // For batched calls (b200_batch.cpp).
    int use_stream(cudaStream_t s);
    int build_walk(const int* ops, int count, int stride, bool pre, std::vector<OpDesc>& tab,
                   std::vector<uint8_t>& dep, bool& idempotent, bool& has_op_cum);
    int build_matrix_jobs(const int* eig, const int* rix, const int* prob, const int* d1,
                          const int* d2, const double* t, int count, std::vector<MatJob>& jobs);
    int build_deriv(const int* post, const int* pre, const int* dmat, const int* cw, int count,
                    std::vector<DerivDesc>& tab);
    friend class Batch;

private:
    bool is_tip(int b) const { return b >= 0 && b < N_; }
    bool buf_ok(int b) const { return b >= 0 && b < nbuf_; }
    bool has_data(int b) const { return buf_ok(b) && (partials_[b] || states_[b]); }
    void* mat(int m) const { return (char*)d_mat_ + (size_t)m * mat_bytes_; }
    void* mat_t(int m) const { return (char*)d_mat_t_ + (size_t)m * mat_bytes_; }
    double* scale(int i) const { return d_scale_ + (size_t)i * Pp_; }
    int ensure_partials(int b);
    int upload_matrix(int m, const double* in, double pad);
    int upload_partials(int b, const double* in, bool replicate);
    int run_matrix_jobs(const std::vector<MatJob>& jobs);
    int post_or_pre(const int* ops, int count, int stride, int cumulative, bool pre);
    int deliver_sums(int count, double* outDerivs, double* outSum, double* outSumSq);
    static constexpr int kNotFused = 1;   // build_prederiv: the list needs the separate calls
    int build_prederiv(const int* ops, int count, const int* post, const int* dmat,
                       const int* cw, std::vector<OpDesc>& tab, std::vector<DerivDesc>& dtab,
                       std::vector<PreDerivOp>& fops, bool& idempotent);
    int queue_edge_derivatives(const int* post, const int* pre, const int* dmat, const int* cw,
                               int count, bool site_values);
    int prederiv_tc(const int* ops, int count, const int* post, const int* pre, const int* dmat,
                    const int* cw, const std::vector<OpDesc>& tab,
                    const std::vector<DerivDesc>& dtab, bool idempotent, double* outSum,
                    double* outSumSq);
    int sync();
    double* stage(size_t n);     // pinned result staging (ASYNCH results)
    Dims dims() const { return Dims{S_, Sg_, P_, Pp_, C_}; }

    int device_ = 0;
    cudaStream_t stream_ = nullptr;        // where work is queued (own or a batch's)
    cudaStream_t own_stream_ = nullptr;
    long flags_ = 0;
    bool dbl_ = true, log_scalers_ = true, invevec_t_ = false, pre_auto_ = false;
    bool tc_used_ = false;                 // tensor-core kernels launched (status to check)
    bool bulk_used_ = false;               // bulk-copy derivative launched (status to check)
    int* h_tc_status_ = nullptr;           // pinned copies of the tensor-core and bulk-copy
                                           // time-out flags
    int N_ = 0, nbuf_ = 0, S_ = 0, Sg_ = 0, P_ = 0, Pp_ = 0, C_ = 0;
    int neig_ = 0, nmat_ = 0, nscale_ = 0;
    size_t rsz_ = 8, part_bytes_ = 0, mat_bytes_ = 0;

    void* d_part_pool_ = nullptr;          // internal partials buffers
    std::vector<void*> partials_;          // per buffer: device partials or null
    std::vector<int*> states_;             // per buffer: device tip states or null
    std::vector<void*> owned_;             // lazily allocated tip buffers
    void* d_mat_ = nullptr;
    void* d_mat_t_ = nullptr;              // transposed images of the matrices
    std::vector<double> mat_pad_;
    double* d_scale_ = nullptr;
    double* d_cube_ = nullptr;             // [eig][S][S][S]
    double* d_evals_ = nullptr;            // [eig][S]
    double* d_rates_ = nullptr;            // [eig][C]
    double* d_catw_ = nullptr;             // [eig][C]
    double* d_freqs_ = nullptr;            // [eig][S]
    double* d_patw_ = nullptr;             // [Pp]
    double* d_site_ = nullptr;             // [Pp] site lnL
    double* d_site1_ = nullptr;            // [Pp] site d1 (edge lnL)
    double* d_site2_ = nullptr;            // [Pp] site d2 (edge lnL)
    std::vector<double> h_catw_, h_freqs_, h_rates_;
    std::vector<char> eig_set_, rates_set_, catw_set_, freqs_set_;
    std::vector<double> h_patw_;
    std::vector<int> partition_start_;     // pattern partitions (empty = one partition)

    void capture_lengths(std::vector<MatJob>& jobs);
    int deliver_lnl(double* out);
    DevBuf t_ops_post_, t_ops_pre_, t_jobs_, t_deriv_, t_idx_, t_ptr_, scratch_, out_, site_d_;
    DevBuf t_cross_;                       // cross-product factors w_c r_c t_b
    DevBuf t_cateig_;                      // eigen system of each category (model categories)
    DevBuf d_maps_, t_tc_maps_;            // TMA tensor maps; per-op map table
    std::vector<TmaMap> h_maps_;
    std::vector<char> map_ok_;
    const TmaMap* tma_map(int entry, const void* base, bool matrix);
    int tc_op_maps(const int* ops, int count, int stride, bool pre);
    DevBuf t_dep_post_, t_dep_pre_;        // per op: reads the previous op's output
    double* h_out_ = nullptr;              // pinned result staging (SYNCH calls)
    size_t h_out_n_ = 0;
    // ASYNCH mode: results copied into pinned chunks and delivered at the next
    // synchronisation point (any getter, waitForPartials, or a synchronous call).
    bool async_ = false;
    struct Pending {
        double* slot;
        double* dst_sum;          // caller arrays for edge-derivative sums (may be null)
        double* dst_sumsq;
        int count;                // edge-derivative branches (0: a log-likelihood)
    };
    int picked_[5] = {-2, -2, -2, -2, -2};
    std::vector<Pending> pending_;
    // A captured graph: its executable, the deliveries its copies feed and the
    // pinned blocks those copies (and its table uploads) use.
    struct GraphRec {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        std::vector<Pending> deliveries;
        std::vector<void*> pinned;
        // branch lengths of the captured transition-matrix updates, read by
        // the graph from d_len (capture order); replaced by
        // launchGraphWithLengths
        double* d_len = nullptr;
        int len_cap = 0;
        std::vector<double> len;
        bool len_all = true;      // every captured update reads d_len
        // launchGraphWithLengths stages the caller's lengths in a ring of
        // pinned slots (allocated at EndCapture), so the caller's buffer is
        // free again when the call returns; slot k is rewritten only after
        // the copy recorded by len_ev[k] has run
        static constexpr int kLenRing = 4;
        double* h_len_ring = nullptr;
        cudaEvent_t len_ev[kLenRing] = {};
        int ring_i = 0;
    };
    std::vector<GraphRec> graphs_;
    GraphRec cap_;
    bool capturing_ = false;
    void defer(const Pending& pd);
    void free_graph(GraphRec& g);
    std::vector<std::pair<double*, size_t>> chunks_;
    size_t chunk_i_ = 0, chunk_off_ = 0;

    double last_lnl_ = 0, last_d1_ = 0, last_d2_ = 0;
};

}  // namespace b200
