// Batched calls over several instances (the beagleB200Batch* entry points):
// many trees / partitions of uneven pattern and state counts evaluated with a
// handful of launches instead of one launch chain per instance.
//
// The members share one CUDA stream for the batch's lifetime, so a batch call
// and any single-instance call stay ordered.  Each batched call validates and
// resolves every member's arguments exactly as the single-instance call does
// (Instance::build_*), then:
//   * transition matrices: one launch per (S, C) group of members;
//   * post- / pre-order walks and edge derivatives: one launch per category
//     count for the 4-state members (k_walk4_batch, k_deriv4_batch); other
//     members run their own single-instance launch on the shared stream;
//   * scale accumulation, root pre-partials, root log-likelihoods and the
//     final derivative sums: one launch for all members;
//   * the fused post-order walk with scaling and root lnL: one launch per
//     category count when every member is a 4-state one (k_post4root_batch).
// Within the walk calls the tensor-core groups' launches run on a second
// stream beside the 4-state groups' (fork / join around them).
#pragma once
#include <cuda_runtime.h>
#include <vector>

#include "b200_instance.h"

namespace b200 {

class Batch {
public:
    ~Batch();
    // Members must share device and precision.  Returns a BeagleReturnCode.
    int create(const std::vector<Instance*>& members);
    int size() const { return (int)m_.size(); }

    int updateTransitionMatrices(const int* eigenIndices, const int* const* probIdx,
                                 const double* const* edgeLengths, const int* counts);
    int updatePartials(const int* const* ops, const int* counts, const int* cumulative,
                       bool pre);
    int accumulateScaleFactors(const int* const* idx, const int* counts, const int* cumulative,
                               int reset);
    int setRootPrePartials(const int* bufs, const int* freqs);
    int rootLogLikelihoods(const int* bufs, const int* cw, const int* sf, const int* cum,
                           double* out);
    int postRoot(const int* const* ops, const int* counts, const int* cumulative,
                 const int* roots, const int* cw, const int* sf, double* out);
    int edgeDerivatives(const int* const* post, const int* const* pre,
                        const int* const* dmat, const int* cw, const int* counts,
                        double* const* sums, double* const* sumsq);
    int preDerivatives(const int* const* ops, const int* counts, const int* const* post,
                       const int* const* dmat, const int* cw, double* const* sums,
                       double* const* sumsq);
    // Wait for the batch's queued work and deliver deferred results.
    int wait();
    // CUDA graph of the calls between beginCapture and endCapture (every
    // member ASYNCH); launchGraph replays it, results at the next wait().
    int beginCapture();
    int endCapture(int* graph);
    int launchGraph(int graph);
    // New branch lengths for the graph's captured matrix updates (count = all
    // of them, in capture order), then launchGraph.
    int launchGraphWithLengths(int graph, const double* lengths, int count);
    // Members back on their own streams.
    void release();

private:
    int sync();
    double* stage(size_t n);
    bool deferred() const;     // every member is ASYNCH: results wait for wait()

    // A result copied to pinned memory, delivered to dst[0 .. n) at wait();
    // member >= 0 also records the value as that member's last lnL.
    struct Pending {
        const double* src;
        double* dst;
        size_t n;
        int member;
    };
    std::vector<Pending> pending_;
    void push_pending(const Pending& pd);   // or into the capture's deliveries
    struct GraphRec {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        std::vector<Pending> deliveries;
        std::vector<std::pair<int, std::vector<Instance::Pending>>> member_deliveries;
        std::vector<void*> pinned;
        // branch lengths of the captured transition-matrix updates, read by
        // the graph from d_len (capture order: members in batch order, each
        // member's lengths in its call order); replaced per launch by
        // launchGraphWithLengths through a ring of pinned staging slots
        double* d_len = nullptr;
        int len_cap = 0;
        std::vector<double> len;
        bool len_all = true;
        static constexpr int kLenRing = 4;
        double* h_len_ring = nullptr;
        cudaEvent_t len_ev[kLenRing] = {};
        int ring_i = 0;
    };
    std::vector<GraphRec> graphs_;
    GraphRec cap_;
    bool capturing_ = false;
    void free_graph(GraphRec& g);
    std::vector<std::pair<double*, size_t>> chunks_;   // pinned staging, reused after wait()
    size_t chunk_i_ = 0, chunk_off_ = 0;

    std::vector<Instance*> m_;
    cudaStream_t stream_ = nullptr;
    // A second stream for the tensor-core groups' launches of a call, so that
    // they run beside the 4-state groups' (fork: it waits for everything the
    // batch's stream has queued; join: the batch's stream waits for it).
    // Under capture the two become parallel branches of the graph.
    cudaStream_t side_ = nullptr;
    cudaEvent_t fork_ev_ = nullptr, join_ev_ = nullptr;
    cudaError_t fork();
    cudaError_t join();
    int device_ = 0;
    bool dbl_ = false;
    DevBuf t_a_, t_b_, t_c_, t_block_, t_out_;   // per-call tables and scratch
    DevBuf t_out2_;                              // derivative sums (root lnL uses t_out_)
};

}  // namespace b200
