// Host side of one B200 instance.  See b200_instance.h.
//
// Every call validates its indices on the host before anything reaches the
// device (the reference GPU implementation does not; out-of-range indices
// there are undefined behaviour), converts caller arrays into the device
// layout, and enqueues work on the instance's stream.  Calls that return
// results synchronise that stream; the others return as soon as the work is
// queued (the caller's arrays have been copied by then).
#include "b200_instance.h"
#include "b200_tune.h"

#include <cmath>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <unordered_map>

namespace b200 {

void assign_slots(const int* ops, int count, int stride, std::vector<OpDesc>& tab);

enum {
    kSuccess = 0, kErrGeneral = -1, kErrOOM = -2, kErrRange = -5, kErrNoImpl = -7,
    kErrFP = -8,
};

// Flag bits (values of libhmsbeagle/beagle.h:132-177).
constexpr long F_SINGLE = 1L << 0, F_DOUBLE = 1L << 1, F_SYNCH = 1L << 2, F_ASYNCH = 1L << 3;
constexpr long F_EIGEN_REAL = 1L << 4, F_EIGEN_COMPLEX = 1L << 5;
constexpr long F_SCALING_MANUAL = 1L << 6, F_SCALING_AUTO = 1L << 7, F_SCALING_ALWAYS = 1L << 8;
constexpr long F_SCALERS_RAW = 1L << 9, F_SCALERS_LOG = 1L << 10;
constexpr long F_VECTOR_NONE = 1L << 12, F_THREADING_NONE = 1L << 14;
constexpr long F_PROCESSOR_GPU = 1L << 16;
constexpr long F_INVEVEC_STANDARD = 1L << 20, F_INVEVEC_TRANSPOSED = 1L << 21;
constexpr long F_FRAMEWORK_CUDA = 1L << 22, F_SCALING_DYNAMIC = 1L << 25;
constexpr long F_PARALLELOPS_GRID = 1L << 29;
constexpr long F_PRE_MANUAL = 1L << 30, F_PRE_AUTO = 1L << 31;

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) {                                   \
            (void)cudaGetLastError();                              \
            return e_ == cudaErrorMemoryAllocation ? kErrOOM : kErrGeneral; \
        }                                                          \
    } while (0)

// Dispatch a templated launcher on the instance precision.
#define LAUNCH(fn, ...) (dbl_ ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

// ------------------------------------------------------------------ DevBuf
cudaError_t DevBuf::reserve(size_t n) {
    if (n <= bytes) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    last.clear();
    size_t want = std::max<size_t>(n, 256);
    want = (want + 255) & ~size_t(255);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e == cudaSuccess) bytes = want;
    return e;
}

// While this thread captures a CUDA graph (Instance::beginCapture), uploads
// copy through pinned blocks that the graph keeps: a captured copy node reads
// its source at every launch.
namespace {
thread_local std::vector<void*>* t_capture_pinned = nullptr;
std::atomic<unsigned> g_graph_epoch{0};
}

std::vector<void*>*& capture_pinned() { return t_capture_pinned; }
void note_graph_launch() { ++g_graph_epoch; }

cudaError_t DevBuf::upload(const void* src, size_t n, cudaStream_t s) {
    cudaError_t e = reserve(n);
    if (e != cudaSuccess) return e;
    const unsigned ep = g_graph_epoch.load();
    if (!t_capture_pinned && epoch == ep && last.size() == n && n > 0 &&
        std::memcmp(last.data(), src, n) == 0)
        return cudaSuccess;
    epoch = ep;
    if (t_capture_pinned) {
        void* h = nullptr;
        e = cudaMallocHost(&h, n);
        if (e != cudaSuccess) return e;
        t_capture_pinned->push_back(h);
        std::memcpy(h, src, n);
        e = cudaMemcpyAsync(ptr, h, n, cudaMemcpyHostToDevice, s);
    } else {
        e = cudaMemcpyAsync(ptr, src, n, cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) last.assign((const uint8_t*)src, (const uint8_t*)src + n);
    return e;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    last.clear();
}

// -------------------------------------------------------------- lifetime
Instance::~Instance() {
    cudaSetDevice(device_);
    if (capturing_) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(stream_, &g);
        if (g) cudaGraphDestroy(g);
        t_capture_pinned = nullptr;
        capturing_ = false;
        (void)cudaGetLastError();
    }
    if (stream_) cudaStreamSynchronize(stream_);
    for (GraphRec& g : graphs_) free_graph(g);
    free_graph(cap_);
    for (void* p : owned_) cudaFree(p);
    void* bufs[] = {d_part_pool_, d_mat_, d_mat_t_, d_scale_, d_cube_, d_evals_, d_rates_,
                    d_catw_, d_freqs_, d_patw_, d_site_, d_site1_, d_site2_};
    for (void* p : bufs)
        if (p) cudaFree(p);
    for (DevBuf* b : {&t_ops_post_, &t_ops_pre_, &t_jobs_, &t_deriv_, &t_idx_, &t_ptr_,
                      &scratch_, &out_, &site_d_, &t_dep_post_, &t_dep_pre_, &t_cross_,
                      &d_maps_, &t_tc_maps_, &t_cateig_})
        b->release();
    if (h_out_) cudaFreeHost(h_out_);
    if (h_tc_status_) cudaFreeHost(h_tc_status_);
    for (auto& c : chunks_) cudaFreeHost(c.first);
    if (own_stream_) cudaStreamDestroy(own_stream_);
}

int Instance::create(int tipCount, int partialsBufferCount, int compactBufferCount,
                     int stateCount, int patternCount, int eigenBufferCount,
                     int matrixBufferCount, int categoryCount, int scaleBufferCount, int device,
                     long pref, long req) {
    if (tipCount < 1 || stateCount < 2 || patternCount < 1 || categoryCount < 1 ||
        eigenBufferCount < 1 || matrixBufferCount < 0 || scaleBufferCount < 0 ||
        partialsBufferCount < 0 || compactBufferCount < 0 ||
        partialsBufferCount + compactBufferCount <= tipCount)
        return kErrRange;
    // Requirements this resource cannot meet.
    const long unsupported = F_EIGEN_COMPLEX | F_SCALING_AUTO | F_SCALING_ALWAYS |
                             F_SCALING_DYNAMIC | (1L << 11) /*SSE*/ | (1L << 24) /*AVX*/ |
                             (1L << 15) /*CPU*/ | (1L << 23) /*OpenCL*/ | (1L << 27) /*FW CPU*/ |
                             (1L << 13) /*OpenMP*/;
    if (req & unsupported) return kErrNoImpl;
    if ((req & F_SINGLE) && (req & F_DOUBLE)) return kErrNoImpl;
    // State counts up to 64 and up to 8 rate categories (one CTA per category
    // in a thread-block cluster for S != 4).
    if (stateCount > 64 || categoryCount > 8) return kErrNoImpl;
    // Precision: a single-precision requirement or preference selects the mixed
    // path (FP32 partials, FP64 matrices formation and reductions).
    dbl_ = !((req & F_SINGLE) || (!(req & F_DOUBLE) && (pref & F_SINGLE)));
    log_scalers_ = ((pref | req) & F_SCALERS_LOG) != 0;
    invevec_t_ = ((pref | req) & F_INVEVEC_TRANSPOSED) != 0;
    pre_auto_ = ((pref | req) & F_PRE_AUTO) != 0;
    async_ = ((pref | req) & F_ASYNCH) != 0;
    flags_ = F_PROCESSOR_GPU | F_FRAMEWORK_CUDA | F_EIGEN_REAL | F_SCALING_MANUAL |
             F_VECTOR_NONE | F_THREADING_NONE | F_PARALLELOPS_GRID |
             (((pref | req) & F_ASYNCH) ? F_ASYNCH : F_SYNCH) |
             (dbl_ ? F_DOUBLE : F_SINGLE) | (log_scalers_ ? F_SCALERS_LOG : F_SCALERS_RAW) |
             (invevec_t_ ? F_INVEVEC_TRANSPOSED : F_INVEVEC_STANDARD) |
             (pre_auto_ ? F_PRE_AUTO : F_PRE_MANUAL);

    device_ = device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        (void)cudaGetLastError();
        return -6;   // BEAGLE_ERROR_NO_RESOURCE
    }
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10 || prop.minor != 0) return -6;   // sm_100 only
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    own_stream_ = stream_;

    N_ = tipCount;
    nbuf_ = partialsBufferCount + compactBufferCount;
    S_ = stateCount;
    Sg_ = (stateCount + 3) / 4 * 4;
    P_ = patternCount;
    Pp_ = (patternCount + kPatternPad - 1) / kPatternPad * kPatternPad;
    C_ = categoryCount;
    neig_ = eigenBufferCount;
    nmat_ = matrixBufferCount;
    nscale_ = scaleBufferCount;
    rsz_ = dbl_ ? 8 : 4;
    part_bytes_ = (size_t)Pp_ * C_ * Sg_ * rsz_;
    mat_bytes_ = (size_t)C_ * Sg_ * Sg_ * rsz_;

    partials_.assign(nbuf_, nullptr);
    states_.assign(nbuf_, nullptr);
    const int ninternal = nbuf_ - N_;
    CK(cudaMalloc(&d_part_pool_, part_bytes_ * ninternal));
    CK(cudaMemsetAsync(d_part_pool_, 0, part_bytes_ * ninternal, stream_));
    for (int b = N_; b < nbuf_; ++b)
        partials_[b] = (char*)d_part_pool_ + part_bytes_ * (size_t)(b - N_);
    if (nmat_ > 0) {
        CK(cudaMalloc(&d_mat_, mat_bytes_ * nmat_));
        CK(cudaMemsetAsync(d_mat_, 0, mat_bytes_ * nmat_, stream_));
        CK(cudaMalloc(&d_mat_t_, mat_bytes_ * nmat_));
        CK(cudaMemsetAsync(d_mat_t_, 0, mat_bytes_ * nmat_, stream_));
    }
    mat_pad_.assign(nmat_, 1.0);
    if (nscale_ > 0) {
        CK(cudaMalloc(&d_scale_, sizeof(double) * Pp_ * nscale_));
        CK(cudaMemsetAsync(d_scale_, 0, sizeof(double) * Pp_ * nscale_, stream_));
    }
    CK(cudaMalloc(&d_cube_, sizeof(double) * (size_t)neig_ * S_ * S_ * S_));
    CK(cudaMalloc(&d_evals_, sizeof(double) * neig_ * S_));
    CK(cudaMalloc(&d_rates_, sizeof(double) * neig_ * C_));
    CK(cudaMalloc(&d_catw_, sizeof(double) * neig_ * C_));
    CK(cudaMalloc(&d_freqs_, sizeof(double) * neig_ * S_));
    CK(cudaMalloc(&d_patw_, sizeof(double) * Pp_));
    CK(cudaMalloc(&d_site_, sizeof(double) * Pp_));
    CK(cudaMalloc(&d_site1_, sizeof(double) * Pp_));
    CK(cudaMalloc(&d_site2_, sizeof(double) * Pp_));
    CK(cudaMemsetAsync(d_site_, 0, sizeof(double) * Pp_, stream_));
    CK(cudaMemsetAsync(d_site1_, 0, sizeof(double) * Pp_, stream_));
    CK(cudaMemsetAsync(d_site2_, 0, sizeof(double) * Pp_, stream_));
    h_catw_.assign((size_t)neig_ * C_, 0.0);
    h_freqs_.assign((size_t)neig_ * S_, 0.0);
    h_rates_.assign((size_t)neig_ * C_, 0.0);
    eig_set_.assign(neig_, 0);
    rates_set_.assign(neig_, 0);
    catw_set_.assign(neig_, 0);
    freqs_set_.assign(neig_, 0);
    // Pattern weights default to 1 (padded patterns weigh 0).
    h_patw_.assign(Pp_, 0.0);
    std::fill(h_patw_.begin(), h_patw_.begin() + P_, 1.0);
    CK(cudaMemcpyAsync(d_patw_, h_patw_.data(), sizeof(double) * Pp_, cudaMemcpyHostToDevice,
                       stream_));
    h_out_n_ = 64;
    CK(cudaMallocHost(&h_out_, sizeof(double) * h_out_n_));
    CK(cudaMallocHost(&h_tc_status_, 2 * sizeof(int)));
    h_tc_status_[0] = h_tc_status_[1] = 0;
    return sync();
}

// A deferred result: delivered at the next sync, or, while capturing, at
// every launch of the captured graph.
void Instance::defer(const Pending& pd) {
    if (capturing_) cap_.deliveries.push_back(pd);
    else pending_.push_back(pd);
}

// Capture the work of the following calls into a CUDA graph instead of
// running it (ASYNCH instances; calls that wait for results are refused while
// capturing).  Call the same sequence once before capturing, so that every
// device table already has its size and contents: a table that changes is
// uploaded through a pinned copy the graph keeps.
int Instance::beginCapture() {
    if (capturing_ || !async_) return kErrGeneral;
    int rc = sync();
    if (rc) return rc;
    cap_ = GraphRec{};
    // room for the branch lengths of the captured matrix updates (allocated
    // before the capture starts: the graph keeps the address)
    cap_.len_cap = 4 * nmat_;
    CK(cudaMalloc(&cap_.d_len, sizeof(double) * cap_.len_cap));
    const cudaError_t e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        free_graph(cap_);
        return kErrGeneral;
    }
    capturing_ = true;
    t_capture_pinned = &cap_.pinned;
    return kSuccess;
}

int Instance::endCapture(int* graph) {
    if (!capturing_ || !graph) return kErrGeneral;
    capturing_ = false;
    t_capture_pinned = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&cap_.exec, g, 0ULL);
    cap_.graph = g;
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        free_graph(cap_);
        return kErrGeneral;
    }
    // the capture-time lengths, which launchGraph replays until
    // launchGraphWithLengths replaces them
    if (!cap_.len.empty()) {
        e = cudaMemcpy(cap_.d_len, cap_.len.data(), sizeof(double) * cap_.len.size(),
                       cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMallocHost(&cap_.h_len_ring,
                               sizeof(double) * cap_.len.size() * GraphRec::kLenRing);
        for (int k = 0; k < GraphRec::kLenRing && e == cudaSuccess; ++k)
            e = cudaEventCreateWithFlags(&cap_.len_ev[k], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            free_graph(cap_);
            return kErrGeneral;
        }
    }
    graphs_.push_back(cap_);
    cap_ = GraphRec{};
    *graph = (int)graphs_.size() - 1;
    return kSuccess;
}

// Replace the branch lengths of the graph's captured transition-matrix
// updates (count = all of them, in capture order), then launch it.  The
// lengths are copied on the host into one of the graph's pinned staging slots
// before this call returns, whatever kind of memory the caller's array is;
// the slot's copy to the device is stream-ordered before the launch.  A slot
// is reused once the copy last queued from it has run (an event wait that
// only blocks when more than kLenRing launches are still queued ahead of it).
int Instance::launchGraphWithLengths(int graph, const double* lengths, int count) {
    if (capturing_ || graph < 0 || graph >= (int)graphs_.size() || !graphs_[graph].exec)
        return kErrRange;
    GraphRec& g = graphs_[graph];
    if (!g.len_all || count != (int)g.len.size() || (count > 0 && !lengths)) return kErrRange;
    if (count > 0) {
        const int k = g.ring_i;
        g.ring_i = (k + 1) % GraphRec::kLenRing;
        CK(cudaEventSynchronize(g.len_ev[k]));
        double* slot = g.h_len_ring + (size_t)k * count;
        std::copy(lengths, lengths + count, slot);
        CK(cudaMemcpyAsync(g.d_len, slot, sizeof(double) * count, cudaMemcpyHostToDevice,
                           stream_));
        CK(cudaEventRecord(g.len_ev[k], stream_));
    }
    return launchGraph(graph);
}

// Launch a captured graph on the instance's stream; its deferred results
// are delivered at the next sync as the captured calls' would be.
int Instance::launchGraph(int graph) {
    if (capturing_ || graph < 0 || graph >= (int)graphs_.size() || !graphs_[graph].exec)
        return kErrRange;
    note_graph_launch();
    CK(cudaGraphLaunch(graphs_[graph].exec, stream_));
    for (const Pending& pd : graphs_[graph].deliveries) pending_.push_back(pd);
    return kSuccess;
}

int Instance::injectKernelTimeout(int which) {
    if (capturing_ || (which != 0 && which != 1)) return kErrRange;
    if (which == 0) {
        CK(tc_raise_status(stream_));
        tc_used_ = true;
    } else {
        CK(bulk_raise_status(stream_));
        bulk_used_ = true;
    }
    return kSuccess;
}

void Instance::free_graph(GraphRec& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    for (void* p : g.pinned) cudaFreeHost(p);
    if (g.d_len) cudaFree(g.d_len);
    for (cudaEvent_t ev : g.len_ev)
        if (ev) cudaEventDestroy(ev);
    if (g.h_len_ring) cudaFreeHost(g.h_len_ring);
    g = GraphRec{};
}

// Queue this instance's work on `s` (a batch's stream) from now on, after
// everything queued so far; nullptr returns to the instance's own stream.
int Instance::use_stream(cudaStream_t s) {
    CK(cudaStreamSynchronize(stream_));
    stream_ = s ? s : own_stream_;
    return kSuccess;
}

int Instance::sync() {
    if (capturing_) return kErrGeneral;   // a wait would break the capture
    if (tc_used_) CK(tc_status_async(h_tc_status_, stream_));
    if (bulk_used_) CK(bulk_status_async(h_tc_status_ + 1, stream_));
    CK(cudaStreamSynchronize(stream_));
    if ((tc_used_ && h_tc_status_[0]) || (bulk_used_ && h_tc_status_[1])) {
        // A kernel gave up waiting on its tensor-core work or bulk copies and
        // computed garbage: report it instead of the results.
        h_tc_status_[0] = h_tc_status_[1] = 0;
        CK(bulk_clear_status(stream_));
        CK(tc_clear_status(stream_));
        pending_.clear();
        chunk_i_ = 0;
        chunk_off_ = 0;
        return kErrGeneral;
    }
    for (const Pending& pd : pending_) {
        if (pd.count == 0) {
            last_lnl_ = pd.slot[0];
        } else {
            if (pd.dst_sum) std::copy(pd.slot, pd.slot + pd.count, pd.dst_sum);
            if (pd.dst_sumsq) std::copy(pd.slot + pd.count, pd.slot + 2 * pd.count, pd.dst_sumsq);
        }
    }
    pending_.clear();
    chunk_i_ = 0;
    chunk_off_ = 0;
    return kSuccess;
}

// n doubles of pinned staging, valid until the next sync(); chunks are kept
// and reused, a new one is allocated only when the queued results outgrow them.
double* Instance::stage(size_t n) {
    if (capturing_) {
        // a captured copy writes here at every launch of the graph
        double* p = nullptr;
        if (cudaMallocHost(&p, sizeof(double) * n) != cudaSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        cap_.pinned.push_back(p);
        return p;
    }
    while (chunk_i_ < chunks_.size() && chunk_off_ + n > chunks_[chunk_i_].second) {
        ++chunk_i_;
        chunk_off_ = 0;
    }
    if (chunk_i_ == chunks_.size()) {
        const size_t sz = std::max<size_t>(n, 1 << 20);
        double* p = nullptr;
        if (cudaMallocHost(&p, sizeof(double) * sz) != cudaSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        chunks_.emplace_back(p, sz);
        chunk_off_ = 0;
    }
    double* r = chunks_[chunk_i_].first + chunk_off_;
    chunk_off_ += n;
    return r;
}

int Instance::waitForPartials() { return sync(); }

// ------------------------------------------------------------ data in / out
int Instance::ensure_partials(int b) {
    if (partials_[b]) return kSuccess;
    void* p = nullptr;
    CK(cudaMalloc(&p, part_bytes_));
    CK(cudaMemsetAsync(p, 0, part_bytes_, stream_));
    owned_.push_back(p);
    partials_[b] = p;
    return kSuccess;
}

int Instance::setTipStates(int tip, const int* in) {
    if (!is_tip(tip) || !in) return kErrRange;
    if (!states_[tip]) {
        void* p = nullptr;
        CK(cudaMalloc(&p, sizeof(int) * Pp_));
        owned_.push_back(p);
        states_[tip] = (int*)p;
    }
    std::vector<int> h(Pp_, S_);
    for (int p = 0; p < P_; ++p) h[p] = (in[p] < S_ && in[p] >= 0) ? in[p] : S_;
    CK(cudaMemcpyAsync(states_[tip], h.data(), sizeof(int) * Pp_, cudaMemcpyHostToDevice,
                       stream_));
    return sync();
}

// Convert caller partials ([C][P][S], or [P][S] replicated over categories)
// into the device layout [Pp][C][Sg] and upload.
int Instance::upload_partials(int b, const double* in, bool replicate) {
    int rc = ensure_partials(b);
    if (rc) return rc;
    const size_t n = (size_t)Pp_ * C_ * Sg_;
    std::vector<double> hd;
    std::vector<float> hf;
    if (dbl_) hd.assign(n, 0.0); else hf.assign(n, 0.0f);
    for (int c = 0; c < C_; ++c)
        for (int p = 0; p < P_; ++p) {
            const double* src = replicate ? in + (size_t)p * S_ : in + ((size_t)c * P_ + p) * S_;
            const size_t dst = ((size_t)p * C_ + c) * Sg_;
            for (int i = 0; i < S_; ++i) {
                if (dbl_) hd[dst + i] = src[i]; else hf[dst + i] = (float)src[i];
            }
        }
    const void* src = dbl_ ? (const void*)hd.data() : (const void*)hf.data();
    CK(cudaMemcpyAsync(partials_[b], src, n * rsz_, cudaMemcpyHostToDevice, stream_));
    return sync();
}

int Instance::setTipPartials(int tip, const double* in) {
    if (!is_tip(tip) || !in) return kErrRange;
    return upload_partials(tip, in, true);
}

int Instance::setPartials(int b, const double* in) {
    if (!buf_ok(b) || !in) return kErrRange;
    return upload_partials(b, in, false);
}

int Instance::setRootPrePartials(const int* bufs, const int* fidx, int count) {
    if (count < 0 || (count > 0 && (!bufs || !fidx))) return kErrRange;
    for (int k = 0; k < count; ++k) {
        const int b = bufs[k], f = fidx[k];
        if (!buf_ok(b) || f < 0 || f >= neig_ || !freqs_set_[f]) return kErrRange;
        int rc = ensure_partials(b);
        if (rc) return rc;
        CK(LAUNCH(launch_fill_root, partials_[b], d_freqs_ + (size_t)f * S_, dims(), stream_));
    }
    return kSuccess;
}

int Instance::getPartials(int b, int scaleIndex, double* out) {
    if (!buf_ok(b) || !partials_[b] || !out) return kErrRange;
    if (scaleIndex != -1 && (scaleIndex < 0 || scaleIndex >= nscale_)) return kErrRange;
    const size_t n = (size_t)Pp_ * C_ * Sg_;
    std::vector<uint8_t> h(n * rsz_);
    CK(cudaMemcpyAsync(h.data(), partials_[b], n * rsz_, cudaMemcpyDeviceToHost, stream_));
    std::vector<double> sc;
    if (scaleIndex != -1) {
        sc.resize(P_);
        CK(cudaMemcpyAsync(sc.data(), scale(scaleIndex), sizeof(double) * P_,
                           cudaMemcpyDeviceToHost, stream_));
    }
    int rc = sync();
    if (rc) return rc;
    for (int c = 0; c < C_; ++c)
        for (int p = 0; p < P_; ++p)
            for (int i = 0; i < S_; ++i) {
                const size_t src = ((size_t)p * C_ + c) * Sg_ + i;
                out[((size_t)c * P_ + p) * S_ + i] =
                    dbl_ ? ((const double*)h.data())[src] : (double)((const float*)h.data())[src];
            }
    // CPU/BeagleCPUImpl.hpp:734-745: the cumulative factors are applied to the
    // first P*S outputs (category 0) only; reproduced as is.
    if (scaleIndex != -1)
        for (int p = 0; p < P_; ++p) {
            const double f = std::exp(sc[p]);
            for (int i = 0; i < S_; ++i) out[(size_t)p * S_ + i] *= f;
        }
    return kSuccess;
}

int Instance::setEigenDecomposition(int e, const double* evec, const double* ivec,
                                    const double* evals) {
    if (e < 0 || e >= neig_ || !evec || !ivec || !evals) return kErrRange;
    // Cube of the products V[i][k] * Vinv[k][j] (CPU/EigenDecompositionCube.hpp:69-100),
    // stored [i][k][j] so that the threads forming consecutive entries (i, j)
    // of a row read consecutive words for each k.
    const size_t S = S_;
    std::vector<double> cube(S * S * S);
    for (size_t i = 0; i < S; ++i)
        for (size_t k = 0; k < S; ++k)
            for (size_t j = 0; j < S; ++j) {
                const double vi = invevec_t_ ? ivec[k + j * S] : ivec[k * S + j];
                cube[(i * S + k) * S + j] = evec[i * S + k] * vi;
            }
    CK(cudaMemcpyAsync(d_cube_ + (size_t)e * S * S * S, cube.data(), sizeof(double) * S * S * S,
                       cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(d_evals_ + (size_t)e * S, evals, sizeof(double) * S,
                       cudaMemcpyHostToDevice, stream_));
    eig_set_[e] = 1;
    return sync();
}

int Instance::setStateFrequencies(int i, const double* f) {
    if (i < 0 || i >= neig_ || !f) return kErrRange;
    std::copy(f, f + S_, h_freqs_.begin() + (size_t)i * S_);
    freqs_set_[i] = 1;
    CK(cudaMemcpyAsync(d_freqs_ + (size_t)i * S_, h_freqs_.data() + (size_t)i * S_,
                       sizeof(double) * S_, cudaMemcpyHostToDevice, stream_));
    return sync();
}

int Instance::setCategoryWeights(int i, const double* w) {
    if (i < 0 || i >= neig_ || !w) return kErrRange;
    std::copy(w, w + C_, h_catw_.begin() + (size_t)i * C_);
    catw_set_[i] = 1;
    CK(cudaMemcpyAsync(d_catw_ + (size_t)i * C_, h_catw_.data() + (size_t)i * C_,
                       sizeof(double) * C_, cudaMemcpyHostToDevice, stream_));
    return sync();
}

int Instance::setCategoryRatesWithIndex(int i, const double* r) {
    if (i < 0 || i >= neig_ || !r) return kErrRange;
    std::copy(r, r + C_, h_rates_.begin() + (size_t)i * C_);
    rates_set_[i] = 1;
    CK(cudaMemcpyAsync(d_rates_ + (size_t)i * C_, h_rates_.data() + (size_t)i * C_,
                       sizeof(double) * C_, cudaMemcpyHostToDevice, stream_));
    return sync();
}

int Instance::setPatternWeights(const double* w) {
    if (!w) return kErrRange;
    std::copy(w, w + P_, h_patw_.begin());
    CK(cudaMemcpyAsync(d_patw_, h_patw_.data(), sizeof(double) * Pp_, cudaMemcpyHostToDevice,
                       stream_));
    return sync();
}

int Instance::setPatternPartitions(int n, const int* parts) {
    // Partitions must be contiguous, ascending pattern ranges here (the
    // reference CPU reorders patterns otherwise, BeagleCPUImpl.hpp:803-920).
    if (n < 1 || !parts) return kErrRange;
    std::vector<int> start(n + 1, -1);
    int cur = parts[0];
    if (cur != 0) return kErrNoImpl;
    start[0] = 0;
    for (int p = 1; p < P_; ++p) {
        if (parts[p] == cur) continue;
        if (parts[p] != cur + 1) return kErrNoImpl;
        cur = parts[p];
        start[cur] = p;
    }
    if (cur != n - 1) return kErrRange;
    start[n] = P_;
    partition_start_ = start;
    return kSuccess;
}

// ---------------------------------------------------------------- matrices
int Instance::upload_matrix(int m, const double* in, double pad) {
    // Natural image [C][Sg][Sg] and its transpose, zero padded.
    const size_t n = (size_t)C_ * Sg_ * Sg_;
    std::vector<double> hd(2 * n, 0.0);
    for (int c = 0; c < C_; ++c)
        for (int i = 0; i < S_; ++i)
            for (int j = 0; j < S_; ++j) {
                const double v = in[((size_t)c * S_ + i) * S_ + j];
                hd[((size_t)c * Sg_ + i) * Sg_ + j] = v;
                hd[n + ((size_t)c * Sg_ + j) * Sg_ + i] = v;
            }
    if (dbl_) {
        CK(cudaMemcpyAsync(mat(m), hd.data(), n * 8, cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync(mat_t(m), hd.data() + n, n * 8, cudaMemcpyHostToDevice, stream_));
    } else {
        std::vector<float> hf(hd.begin(), hd.end());
        CK(cudaMemcpyAsync(mat(m), hf.data(), n * 4, cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync(mat_t(m), hf.data() + n, n * 4, cudaMemcpyHostToDevice, stream_));
        mat_pad_[m] = pad;
        return sync();   // hf goes out of scope
    }
    mat_pad_[m] = pad;
    return sync();
}

int Instance::setTransitionMatrix(int m, const double* in, double pad) {
    if (m < 0 || m >= nmat_ || !in) return kErrRange;
    int rc = upload_matrix(m, in, pad);
    mat_pad_[m] = pad;
    return rc;
}

int Instance::setTransitionMatrices(const int* idx, const double* in, const double* pads,
                                    int count) {
    for (int k = 0; k < count; ++k) {
        int rc = setTransitionMatrix(idx[k], in + (size_t)k * C_ * S_ * S_, pads[k]);
        if (rc) return rc;
    }
    return kSuccess;
}

int Instance::getTransitionMatrix(int m, double* out) {
    if (m < 0 || m >= nmat_ || !out) return kErrRange;
    const size_t n = (size_t)C_ * Sg_ * Sg_;
    std::vector<uint8_t> h(n * rsz_);
    CK(cudaMemcpyAsync(h.data(), mat(m), n * rsz_, cudaMemcpyDeviceToHost, stream_));
    int rc = sync();
    if (rc) return rc;
    for (int c = 0; c < C_; ++c)
        for (int i = 0; i < S_; ++i)
            for (int j = 0; j < S_; ++j) {
                const size_t src = ((size_t)c * Sg_ + i) * Sg_ + j;
                out[((size_t)c * S_ + i) * S_ + j] =
                    dbl_ ? ((const double*)h.data())[src] : (double)((const float*)h.data())[src];
            }
    return kSuccess;
}

int Instance::transposeTransitionMatrices(const int* in, const int* out, int count) {
    if (count <= 0) return kSuccess;
    // pointer table: inputs, results, results' transposed images
    std::vector<const void*> tab(3 * count);
    for (int k = 0; k < count; ++k) {
        if (in[k] < 0 || in[k] >= nmat_ || out[k] < 0 || out[k] >= nmat_) return kErrRange;
        if (in[k] == out[k]) return kErrRange;   // in-place not allowed (CPU :1190-1200)
        tab[k] = mat(in[k]);
        tab[count + k] = mat(out[k]);
        tab[2 * count + k] = mat_t(out[k]);
    }
    CK(t_ptr_.upload(tab.data(), sizeof(void*) * tab.size(), stream_));
    const void* const* base = (const void* const*)t_ptr_.ptr;
    CK(LAUNCH(launch_matrix_pairs, base, nullptr, (void* const*)(base + count), count, 1, dims(),
              stream_));
    return kSuccess;
}

int Instance::convolveTransitionMatrices(const int* first, const int* second,
                                         const int* result, int count) {
    if (count <= 0) return kSuccess;
    // pointer table: first, second, results, results' transposed images
    std::vector<const void*> tab(4 * count);
    for (int k = 0; k < count; ++k) {
        for (int v : {first[k], second[k], result[k]})
            if (v < 0 || v >= nmat_) return kErrRange;
        if (first[k] == result[k] || second[k] == result[k]) return kErrRange;
        tab[k] = mat(first[k]);
        tab[count + k] = mat(second[k]);
        tab[2 * count + k] = mat(result[k]);
        tab[3 * count + k] = mat_t(result[k]);
        mat_pad_[result[k]] = 1.0;
    }
    CK(t_ptr_.upload(tab.data(), sizeof(void*) * tab.size(), stream_));
    const void* const* base = (const void* const*)t_ptr_.ptr;
    CK(LAUNCH(launch_matrix_pairs, base, base + count, (void* const*)(base + 2 * count), count, 0,
              dims(), stream_));
    return kSuccess;
}

int Instance::run_matrix_jobs(const std::vector<MatJob>& jobs) {
    if (jobs.empty()) return kSuccess;
    CK(t_jobs_.upload(jobs.data(), sizeof(MatJob) * jobs.size(), stream_));
    CK(LAUNCH(launch_update_matrices, (const MatJob*)t_jobs_.ptr, (int)jobs.size(), dims(),
              stream_));
    return kSuccess;
}

int Instance::updateTransitionMatricesWithMultipleModels(const int* eig, const int* rix,
                                                         const int* prob, const int* d1,
                                                         const int* d2, const double* t,
                                                         int count) {
    std::vector<MatJob> jobs;
    const int rc = build_matrix_jobs(eig, rix, prob, d1, d2, t, count, jobs);
    if (rc) return rc;
    capture_lengths(jobs);
    return run_matrix_jobs(jobs);
}

// While capturing, the jobs read their branch lengths from the graph's
// lengths buffer (capture order), so that launchGraphWithLengths can replace
// them; past the buffer's room they keep the captured values.
void Instance::capture_lengths(std::vector<MatJob>& jobs) {
    if (!capturing_ || !cap_.d_len) return;
    if ((int)(cap_.len.size() + jobs.size()) > cap_.len_cap) {
        cap_.len_all = false;
        return;
    }
    for (MatJob& j : jobs) {
        j.tlen = cap_.d_len + cap_.len.size();
        cap_.len.push_back(j.t);
    }
}

// Validate and resolve transition-matrix requests into device jobs.
int Instance::build_matrix_jobs(const int* eig, const int* rix, const int* prob, const int* d1,
                                const int* d2, const double* t, int count,
                                std::vector<MatJob>& jobs) {
    if (count < 0 || (count > 0 && (!prob || !t))) return kErrRange;
    jobs.assign(count, MatJob{});
    for (int u = 0; u < count; ++u) {
        const int e = eig ? eig[u] : 0, r = rix ? rix[u] : 0;
        if (e < 0 || e >= neig_ || !eig_set_[e] || r < 0 || r >= neig_ || !rates_set_[r])
            return kErrRange;
        if (prob[u] < 0 || prob[u] >= nmat_) return kErrRange;
        if (d1 && (d1[u] < 0 || d1[u] >= nmat_)) return kErrRange;
        if (d2 && (d2[u] < 0 || d2[u] >= nmat_)) return kErrRange;
        MatJob& j = jobs[u];
        j.p = mat(prob[u]);
        j.d1 = d1 ? mat(d1[u]) : nullptr;
        j.d2 = (d1 && d2) ? mat(d2[u]) : nullptr;
        j.pt = mat_t(prob[u]);
        j.d1t = d1 ? mat_t(d1[u]) : nullptr;
        j.d2t = (d1 && d2) ? mat_t(d2[u]) : nullptr;
        j.cube = d_cube_ + (size_t)e * S_ * S_ * S_;
        j.evals = d_evals_ + (size_t)e * S_;
        j.rates = d_rates_ + (size_t)r * C_;
        j.t = t[u];
        j.tlen = nullptr;
        mat_pad_[prob[u]] = 1.0;
        if (j.d1) mat_pad_[d1[u]] = 0.0;
        if (j.d2) mat_pad_[d2[u]] = 0.0;
    }
    return kSuccess;
}

int Instance::updateTransitionMatrices(int e, const int* prob, const int* d1, const int* d2,
                                       const double* t, int count) {
    std::vector<int> eig(std::max(count, 0), e), rix(std::max(count, 0), 0);
    return updateTransitionMatricesWithMultipleModels(eig.data(), rix.data(), prob, d1, d2, t,
                                                      count);
}

// CPU/EigenDecompositionCube.hpp:326-470: category c of every listed matrix
// from eigen system eig[c], exp(lambda t) without a category rate.
int Instance::updateTransitionMatricesWithModelCategories(const int* eig, const int* prob,
                                                          const int* d1, const int* d2,
                                                          const double* t, int count) {
    if (count < 0 || (count > 0 && !eig)) return kErrRange;
    if (count == 0) return kSuccess;
    for (int c = 0; c < C_; ++c)
        if (eig[c] < 0 || eig[c] >= neig_ || !eig_set_[eig[c]]) return kErrRange;
    std::vector<MatJob> jobs;
    const int rc = build_matrix_jobs(nullptr, nullptr, prob, d1, d2, t, count, jobs);
    if (rc) return rc;
    CK(t_cateig_.upload(eig, sizeof(int) * C_, stream_));
    for (MatJob& j : jobs) {
        j.cube = d_cube_;
        j.evals = d_evals_;
        j.cat_eig = (const int*)t_cateig_.ptr;
    }
    capture_lengths(jobs);
    return run_matrix_jobs(jobs);
}

// ---------------------------------------------------------------- partials
// Validate an op list (7 ints, or 9 for partition ops) and resolve it into
// device descriptors.  dep[k] != 0 when op k reads op k - 1's output;
// `idempotent`: the list may be run again (no op reads a buffer the list
// writes at or after it); `has_op_cum`: some partition op adds into its own
// cumulative buffer.
int Instance::build_walk(const int* ops, int count, int stride, bool pre, std::vector<OpDesc>& tab,
                         std::vector<uint8_t>& dep, bool& idempotent, bool& has_op_cum) {
    if (count < 0 || (count > 0 && !ops)) return kErrRange;
    tab.assign(count, OpDesc{});
    dep.assign(count, 0);
    has_op_cum = false;
    // Buffers written earlier in this list count as holding data.
    std::vector<char> written(nbuf_, 0);
    idempotent = true;
    std::vector<char> later(nbuf_, 0), later_scale(nscale_ > 0 ? nscale_ : 1, 0);
    for (int k = count - 1; k >= 0; --k) {
        const int* op = ops + (size_t)k * stride;
        if (!buf_ok(op[0]) || !buf_ok(op[3]) || !buf_ok(op[5])) break;   // rejected below
        later[op[0]] = 1;
        if (op[1] >= 0 && op[1] < nscale_) later_scale[op[1]] = 1;
        if (later[op[3]] || later[op[5]]) idempotent = false;
        if (op[1] < 0 && op[2] >= 0 && op[2] < nscale_ && later_scale[op[2]]) idempotent = false;
    }
    for (int k = 0; k < count; ++k) {
        const int* op = ops + (size_t)k * stride;
        const int dest = op[0], ws = op[1], rs = op[2], c1 = op[3], m1 = op[4], c2 = op[5],
                  m2 = op[6];
        if (!buf_ok(dest) || states_[dest]) return kErrRange;
        if (!buf_ok(c1) || !buf_ok(c2)) return kErrRange;
        if (!(has_data(c1) || written[c1]) || !(has_data(c2) || written[c2])) return kErrRange;
        if (pre && states_[c1]) return kErrRange;   // parent pre-partials are partials
        if (m1 < 0 || m1 >= nmat_ || m2 < 0 || m2 >= nmat_) return kErrRange;
        if (ws != -1 && (ws < 0 || ws >= nscale_)) return kErrRange;
        if (rs != -1 && (rs < 0 || rs >= nscale_)) return kErrRange;
        if (dest == c1 || dest == c2) return kErrRange;
        int rc = ensure_partials(dest);
        if (rc) return rc;
        written[dest] = 1;
        OpDesc& d = tab[k];
        d.x1 = states_[c1] ? (const void*)states_[c1] : partials_[c1];
        d.x2 = states_[c2] ? (const void*)states_[c2] : partials_[c2];
        d.dest = partials_[dest];
        d.m1 = mat(m1);
        d.m2 = mat(m2);
        d.m1t = mat_t(m1);
        d.m2t = mat_t(m2);
        if (k > 0 && (c1 == ops[(size_t)(k - 1) * stride] || c2 == ops[(size_t)(k - 1) * stride]))
            dep[k] = 1;
        d.pad1 = mat_pad_[m1];
        d.pad2 = mat_pad_[m2];
        d.scale_write = ws >= 0 ? scale(ws) : nullptr;
        // Fixed scaling applies only when no new factors are written
        // (CPU/BeagleCPUImpl.hpp:1571-1577); pre-order never reads them (:1779-1785).
        d.scale_read = (ws < 0 && rs >= 0 && !pre) ? scale(rs) : nullptr;
        d.kind = (states_[c1] ? kX1States : 0) | (states_[c2] ? kX2States : 0);
        // The reference GPU resource expects the node's matrix transposed in
        // pre-order ops when S > 4 unless PREORDER_TRANSPOSE_AUTO is set
        // (GPU/BeagleGPUImpl.hpp:787-788, 2844-2855).
        if (pre && S_ > 4 && !pre_auto_) d.kind |= kM1Transposed;
        d.p_begin = 0;
        d.p_end = Pp_;
        d.cum = nullptr;
        if (stride == 9) {
            // Partition op (beagle.h:922-932): the partition's pattern range and
            // its own cumulative scale buffer (CPU/BeagleCPUImpl.hpp:1527-1534).
            const int part = op[7], pcum = op[8];
            if (partition_start_.empty() || part < 0 ||
                part >= (int)partition_start_.size() - 1)
                return kErrRange;
            if (pcum != -1 && (pcum < 0 || pcum >= nscale_)) return kErrRange;
            d.p_begin = partition_start_[part];
            d.p_end = partition_start_[part + 1];
            if (pcum >= 0 && !pre) {
                d.cum = scale(pcum);
                has_op_cum = true;
            }
        }
        d.slots = 0;
    }
    if (stride == 7) assign_slots(ops, count, stride, tab);
    return kSuccess;
}

// Shared-memory slots for the S = 4 slot walks: a linear scan over the list
// gives each result that a later op reads one of kMaxSlots slots, from its op
// to its last reader (a buffer rewritten later in the list starts a new value);
// results that find no free slot are read back from device memory as usual.
void assign_slots(const int* ops, int count, int stride, std::vector<OpDesc>& tab) {
    std::unordered_map<int, int> producer;          // buffer -> op that wrote its value
    std::vector<int> src1(count, -1), src2(count, -1), last(count, -1);
    for (int k = 0; k < count; ++k) {
        const int* op = ops + (size_t)k * stride;
        auto it = producer.find(op[3]);
        if (it != producer.end()) src1[k] = it->second, last[it->second] = k;
        it = producer.find(op[5]);
        if (it != producer.end()) src2[k] = it->second, last[it->second] = k;
        producer[op[0]] = k;
    }
    std::vector<int> slot(count, -1), free_slots;
    std::vector<std::vector<int>> ends(count);
    for (int s = kMaxSlots - 1; s >= 0; --s) free_slots.push_back(s);
    for (int k = 0; k < count; ++k) {
        for (int j : ends[k]) free_slots.push_back(slot[j]);   // op k reads, then writes
        if (last[k] > k && !free_slots.empty()) {
            slot[k] = free_slots.back();
            free_slots.pop_back();
            ends[last[k]].push_back(k);
        }
    }
    for (int k = 0; k < count; ++k) {
        const int in1 = src1[k] >= 0 ? slot[src1[k]] : -1;
        const int in2 = src2[k] >= 0 ? slot[src2[k]] : -1;
        tab[k].slots = (slot[k] + 1) | ((in1 + 1) << 4) | ((in2 + 1) << 8);
    }
}

// TMA tensor map of partials buffer b (entry b) or of matrix m (entry nbuf + m)
// in a device array created once; encoded and copied on first use.
const TmaMap* Instance::tma_map(int entry, const void* base, bool matrix) {
    const size_t n = (size_t)nbuf_ + 2 * (size_t)nmat_;
    if (h_maps_.empty()) {
        if (d_maps_.reserve(sizeof(TmaMap) * n) != cudaSuccess) return nullptr;
        h_maps_.resize(n);
        map_ok_.assign(n, 0);
    }
    TmaMap* dev = (TmaMap*)d_maps_.ptr + entry;
    if (!map_ok_[entry]) {
        if (tc_encode_map(&h_maps_[entry], base, matrix, dims()) != cudaSuccess) return nullptr;
        const void* src = &h_maps_[entry];
        if (capture_pinned()) {   // a captured copy reads its source at every launch
            void* h = nullptr;
            if (cudaMallocHost(&h, sizeof(TmaMap)) != cudaSuccess) return nullptr;
            capture_pinned()->push_back(h);
            std::memcpy(h, src, sizeof(TmaMap));
            src = h;
        }
        if (cudaMemcpyAsync(dev, src, sizeof(TmaMap), cudaMemcpyHostToDevice, stream_) !=
            cudaSuccess)
            return nullptr;
        map_ok_[entry] = 1;
    }
    return dev;
}

// Per-op tensor maps of a walk (TcOpMaps into t_tc_maps_): post-order, both
// children and their matrices; pre-order, the sibling and its matrix (a2,
// b2) and the image of the node's matrix that the second product reads as
// rows of P_node^T (b1): the op's matrix itself when it is given transposed
// (kM1Transposed), else its transposed image (entries nbuf + nmat + m).
int Instance::tc_op_maps(const int* ops, int count, int stride, bool pre) {
    std::vector<TcOpMaps> tab(count);
    const bool given_transposed = S_ > 4 && !pre_auto_;
    for (int k = 0; k < count; ++k) {
        const int* op = ops + (size_t)k * stride;
        TcOpMaps& m = tab[k];
        m = TcOpMaps{nullptr, nullptr, nullptr, nullptr};
        auto part = [&](int b) -> const TmaMap* {
            return states_[b] ? nullptr : tma_map(b, partials_[b], false);
        };
        if (!pre && !states_[op[3]]) {
            m.a1 = part(op[3]);
            m.b1 = tma_map(nbuf_ + op[4], mat(op[4]), true);
            if (!m.a1 || !m.b1) return kErrGeneral;
        }
        if (!states_[op[5]]) {
            m.a2 = part(op[5]);
            m.b2 = tma_map(nbuf_ + op[6], mat(op[6]), true);
            if (!m.a2 || !m.b2) return kErrGeneral;
        }
        if (pre) {
            m.b1 = given_transposed ? tma_map(nbuf_ + op[4], mat(op[4]), true)
                                    : tma_map(nbuf_ + nmat_ + op[4], mat_t(op[4]), true);
            if (!m.b1) return kErrGeneral;
        }
    }
    CK(t_tc_maps_.upload(tab.data(), sizeof(TcOpMaps) * count, stream_));
    return kSuccess;
}

int Instance::post_or_pre(const int* ops, int count, int stride, int cumulative, bool pre) {
    if (cumulative != -1 && (cumulative < 0 || cumulative >= nscale_)) return kErrRange;
    std::vector<OpDesc> tab;
    std::vector<uint8_t> dep;
    bool idempotent = true, has_op_cum = false;
    int rc = build_walk(ops, count, stride, pre, tab, dep, idempotent, has_op_cum);
    if (rc) return rc;
    if (count == 0) return kSuccess;
    DevBuf& t = pre ? t_ops_pre_ : t_ops_post_;
    CK(t.upload(tab.data(), sizeof(OpDesc) * tab.size(), stream_));
    double* cum = (cumulative >= 0 && !pre) ? scale(cumulative) : nullptr;
    if (S_ != 4) {
        DevBuf& td = pre ? t_dep_pre_ : t_dep_post_;
        CK(td.upload(dep.data(), dep.size(), stream_));
        const OpDesc* d_ops = (const OpDesc*)t.ptr;
        const Dims dm = dims();
        const int ls = (int)log_scalers_;
        // variant 0: CUDA-core cluster kernels; 1: tensor cores (FP32 only);
        // 2: tensor cores fed by TMA (FP32 only)
        auto run = [&](int v) -> cudaError_t {
            if (v == 2) {
                if (tc_op_maps(ops, count, stride, pre) != kSuccess) return cudaErrorInvalidValue;
                tc_used_ = true;
                return launch_opwalk_tc_tma(d_ops, (const TcOpMaps*)t_tc_maps_.ptr, count, pre,
                                            dm, cum, ls, stream_);
            }
            if (v == 1) {
                tc_used_ = true;
                return launch_opwalk_tc(d_ops, count, pre, dm, cum, ls, stream_);
            }
            return LAUNCH(launch_opwalk_generic, d_ops, (const uint8_t*)td.ptr, count, pre, dm,
                          cum, ls, stream_);
        };
        const bool tc = !dbl_ && tc_supported(dm);
        const TuneKey key{pre ? kTuneWalkPre : kTuneWalkPost, (int)dbl_, C_ * 100 + Sg_, Pp_,
                          tune_count_class(count), device_};
        int v = tune_pick(key, tc ? 3 : 1, idempotent && !cum && !has_op_cum, stream_, run);
        if (v < 0) v = tc ? 1 : 0;
        cudaError_t e = run(v);
        if ((e == cudaErrorInvalidConfiguration || e == cudaErrorInvalidValue) && v >= 1) {
            (void)cudaGetLastError();
            v = 0;
            e = run(0);
        }
        picked_[pre ? kTuneWalkPre : kTuneWalkPost] = v;
        CK(e);
    } else {
        const OpDesc* d_ops = (const OpDesc*)t.ptr;
        const Dims dm = dims();
        const int ls = (int)log_scalers_;
        const bool ranged = stride == 9;
        const OpDesc* h_ops = tab.data();
        auto run = [&](int v) -> cudaError_t {
            return pre ? LAUNCH(launch_update_pre_partials, d_ops, count, dm, ls, stream_, v,
                                ranged, h_ops)
                       : LAUNCH(launch_update_partials, d_ops, count, dm, cum, ls, stream_, v,
                                ranged, h_ops);
        };
        const TuneKey key{pre ? kTuneWalkPre : kTuneWalkPost, (int)dbl_, C_, Pp_,
                          tune_count_class(count), device_};
        const int v = tune_pick(key, s4_walk_variants(C_), idempotent && !cum && !has_op_cum,
                                stream_, run);
        picked_[pre ? kTuneWalkPre : kTuneWalkPost] = v;
        CK(run(v));
    }
    return kSuccess;
}

int Instance::updatePartials(const int* ops, int count, int cumulative) {
    return post_or_pre(ops, count, 7, cumulative, false);
}

int Instance::updatePrePartials(const int* ops, int count, int cumulative) {
    return post_or_pre(ops, count, 7, cumulative, true);
}

// Partition ops (9 ints) run as one launch over the whole list, each op
// writing only its partition's patterns (CPU/BeagleCPUImpl.hpp:1395-1434).
int Instance::updatePartialsByPartition(const int* ops, int count) {
    return post_or_pre(ops, count, 9, -1, false);
}

int Instance::updatePrePartialsByPartition(const int* ops, int count) {
    return post_or_pre(ops, count, 9, -1, true);
}

// ------------------------------------------------------------ scale factors
int Instance::accumulateScaleFactors(const int* idx, int count, int cumulative, double sign,
                                     int partition) {
    if (cumulative < 0 || cumulative >= nscale_ || count < 0 || (count > 0 && !idx))
        return kErrRange;
    for (int k = 0; k < count; ++k)
        if (idx[k] < 0 || idx[k] >= nscale_) return kErrRange;
    int p0 = 0, p1 = P_;
    if (partition >= 0) {
        if (partition_start_.empty() || partition >= (int)partition_start_.size() - 1)
            return kErrRange;
        p0 = partition_start_[partition];
        p1 = partition_start_[partition + 1];
    }
    CK(t_idx_.upload(idx, sizeof(int) * count, stream_));
    CK(launch_accumulate_scale(scale(cumulative), d_scale_, (const int*)t_idx_.ptr, count, Pp_,
                               P_, sign, (int)log_scalers_, p0, p1, stream_));
    return kSuccess;
}

int Instance::resetScaleFactors(int cumulative, int partition) {
    if (cumulative < 0 || cumulative >= nscale_) return kErrRange;
    if (partition < 0) {
        CK(cudaMemsetAsync(scale(cumulative), 0, sizeof(double) * Pp_, stream_));
    } else {
        if (partition_start_.empty() || partition >= (int)partition_start_.size() - 1)
            return kErrRange;
        const int p0 = partition_start_[partition], p1 = partition_start_[partition + 1];
        CK(cudaMemsetAsync(scale(cumulative) + p0, 0, sizeof(double) * (p1 - p0), stream_));
    }
    return kSuccess;
}

int Instance::copyScaleFactors(int dst, int src) {
    if (dst < 0 || dst >= nscale_ || src < 0 || src >= nscale_) return kErrRange;
    CK(cudaMemcpyAsync(scale(dst), scale(src), sizeof(double) * Pp_, cudaMemcpyDeviceToDevice,
                       stream_));
    return kSuccess;
}

int Instance::getScaleFactors(int src, double* out) {
    if (src < 0 || src >= nscale_ || !out) return kErrRange;
    CK(cudaMemcpyAsync(out, scale(src), sizeof(double) * P_, cudaMemcpyDeviceToHost, stream_));
    return sync();
}

// -------------------------------------------------------------- reductions
int Instance::calculateRootLogLikelihoods(const int* bufs, const int* cw, const int* sf,
                                          const int* cum, int count, double* out) {
    if (count != 1) return kErrNoImpl;
    if (!bufs || !cw || !sf || !out) return kErrRange;
    const int b = bufs[0], w = cw[0], f = sf[0], c = cum ? cum[0] : -1;
    if (!buf_ok(b) || !partials_[b]) return kErrRange;
    if (w < 0 || w >= neig_ || !catw_set_[w] || f < 0 || f >= neig_ || !freqs_set_[f])
        return kErrRange;
    if (c != -1 && (c < 0 || c >= nscale_)) return kErrRange;
    const int nblk = root_blocks(dims(), P_, true);
    CK(scratch_.reserve(sizeof(double) * nblk));
    CK(out_.reserve(sizeof(double) * 4));
    CK(LAUNCH(launch_root_lnl, partials_[b], d_catw_ + (size_t)w * C_, d_freqs_ + (size_t)f * S_,
              c >= 0 ? scale(c) : nullptr, d_patw_, dims(), d_site_, (double*)scratch_.ptr,
              (double*)out_.ptr, stream_));
    return deliver_lnl(out);
}

// The lnL in out_[0] to the caller: now, or (ASYNCH, GPU/BeagleGPUImpl.hpp:
// 3398-3407) at beagleGetLogLikelihood, with nothing written to *out here.
int Instance::deliver_lnl(double* out) {
    if (async_) {
        double* slot = stage(1);
        if (!slot) return kErrOOM;
        CK(cudaMemcpyAsync(slot, out_.ptr, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        defer(Pending{slot, nullptr, nullptr, 0});
        return kSuccess;
    }
    CK(cudaMemcpyAsync(h_out_, out_.ptr, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    int rc = sync();
    if (rc) return rc;
    *out = h_out_[0];
    last_lnl_ = *out;
    return std::isnan(*out) ? kErrFP : kSuccess;
}

// updatePartials(ops, count, NONE); with a cumulative buffer, resetScaleFactors
// on it and accumulateScaleFactors of the list's scale buffers; then
// calculateRootLogLikelihoods of `root` -- in one launch (k_post4root) when
// the root is the last op's destination and the list is a plain S = 4 one
// of at most 256 ops, otherwise as those calls.
int Instance::updatePartialsWithRootLogLikelihood(const int* ops, int count, int cumulative,
                                                  int root, int cw, int sf, double* out) {
    if (!out) return kErrRange;
    if (cumulative != -1 && (cumulative < 0 || cumulative >= nscale_)) return kErrRange;
    std::vector<int> written;
    for (int k = 0; ops && k < count; ++k)
        if (ops[(size_t)k * 7 + 1] >= 0) written.push_back(ops[(size_t)k * 7 + 1]);
    auto separate = [&]() -> int {
        int rc = updatePartials(ops, count, -1);
        if (rc) return rc;
        if (cumulative >= 0) {
            rc = resetScaleFactors(cumulative, -1);
            if (rc) return rc;
            rc = accumulateScaleFactors(written.data(), (int)written.size(), cumulative, 1.0, -1);
            if (rc) return rc;
        }
        const int* cp = cumulative >= 0 ? &cumulative : nullptr;
        return calculateRootLogLikelihoods(&root, &cw, &sf, cp, 1, out);
    };
    bool fused = S_ == 4 && (C_ == 1 || C_ == 2 || C_ == 4 || C_ == 8) && count >= 1 &&
                 count <= 256 && ops && ops[(size_t)(count - 1) * 7] == root;
    for (int k = 0; fused && k < (int)written.size(); ++k)
        if (written[k] == cumulative) fused = false;   // the list rewrites the cumulative buffer
    if (!fused) return separate();
    if (!buf_ok(root) || cw < 0 || cw >= neig_ || !catw_set_[cw] || sf < 0 || sf >= neig_ ||
        !freqs_set_[sf])
        return kErrRange;
    std::vector<OpDesc> tab;
    std::vector<uint8_t> dep;
    bool idempotent = true, has_op_cum = false;
    int rc = build_walk(ops, count, 7, false, tab, dep, idempotent, has_op_cum);
    if (rc) return rc;
    const Dims dm = dims();
    CK(scratch_.reserve(sizeof(double) * post_root_blocks(dm)));
    CK(out_.reserve(sizeof(double) * 4));
    CK(LAUNCH(launch_post4_root, tab.data(), count, dm, cumulative >= 0 ? scale(cumulative) : nullptr,
              (int)log_scalers_, d_catw_ + (size_t)cw * C_, d_freqs_ + (size_t)sf * S_, d_patw_,
              d_site_, (double*)scratch_.ptr, (double*)out_.ptr, stream_));
    picked_[kTuneWalkPost] = 7;
    return deliver_lnl(out);
}

// CPU/BeagleCPUImpl.hpp:2349-2388: one root per partition (count == 1), the
// lnL of each partition over its patterns and their total.
int Instance::calculateRootLogLikelihoodsByPartition(const int* bufs, const int* cw,
                                                     const int* sf, const int* cum,
                                                     const int* parts, int nparts, int count,
                                                     double* outByPart, double* out) {
    if (count != 1) return kErrNoImpl;
    if (nparts < 1 || !bufs || !cw || !sf || !parts || !outByPart || !out) return kErrRange;
    if (partition_start_.empty()) return kErrRange;
    const int npart_defined = (int)partition_start_.size() - 1;
    int total_blocks = 0;
    for (int i = 0; i < nparts; ++i) {
        const int b = bufs[i], w = cw[i], f = sf[i], c = cum ? cum[i] : -1, q = parts[i];
        if (!buf_ok(b) || !partials_[b]) return kErrRange;
        if (w < 0 || w >= neig_ || !catw_set_[w] || f < 0 || f >= neig_ || !freqs_set_[f])
            return kErrRange;
        if (c != -1 && (c < 0 || c >= nscale_)) return kErrRange;
        if (q < 0 || q >= npart_defined) return kErrRange;
        total_blocks += root_blocks(dims(), partition_start_[q + 1] - partition_start_[q], true);
    }
    CK(scratch_.reserve(sizeof(double) * std::max(total_blocks, 1)));
    CK(out_.reserve(sizeof(double) * std::max(nparts, 4)));
    double* blocks = (double*)scratch_.ptr;
    for (int i = 0; i < nparts; ++i) {
        const int b = bufs[i], w = cw[i], f = sf[i], c = cum ? cum[i] : -1, q = parts[i];
        const int p0 = partition_start_[q], p1 = partition_start_[q + 1];
        CK(LAUNCH(launch_root_lnl_range, partials_[b], d_catw_ + (size_t)w * C_,
                  d_freqs_ + (size_t)f * S_, c >= 0 ? scale(c) : nullptr, d_patw_, dims(), p0, p1,
                  d_site_, blocks, (double*)out_.ptr + i, stream_));
        blocks += root_blocks(dims(), p1 - p0, true);
    }
    if ((size_t)nparts > h_out_n_) {
        cudaFreeHost(h_out_);
        h_out_ = nullptr;
        h_out_n_ = nparts;
        CK(cudaMallocHost(&h_out_, sizeof(double) * h_out_n_));
    }
    CK(cudaMemcpyAsync(h_out_, out_.ptr, sizeof(double) * nparts, cudaMemcpyDeviceToHost,
                       stream_));
    int rc = sync();
    if (rc) return rc;
    double total = 0;
    for (int i = 0; i < nparts; ++i) {
        outByPart[i] = h_out_[i];
        total += h_out_[i];
    }
    *out = total;
    last_lnl_ = total;
    return std::isnan(total) ? kErrFP : kSuccess;
}

// Validate and resolve an edge-derivative request into device descriptors.
int Instance::build_deriv(const int* post, const int* pre, const int* dmat, const int* cw,
                          int count, std::vector<DerivDesc>& tab) {
    if (count < 0 || (count > 0 && (!post || !pre || !dmat || !cw))) return kErrRange;
    if (count == 0) return kSuccess;
    const int w = cw[0];
    if (w < 0 || w >= neig_ || !catw_set_[w]) return kErrRange;
    tab.assign(count, DerivDesc{});
    for (int k = 0; k < count; ++k) {
        if (!has_data(post[k]) || !buf_ok(pre[k]) || !partials_[pre[k]]) return kErrRange;
        if (dmat[k] < 0 || dmat[k] >= nmat_) return kErrRange;
        DerivDesc& d = tab[k];
        d.post = states_[post[k]] ? (const void*)states_[post[k]] : partials_[post[k]];
        d.post_is_states = states_[post[k]] ? 1 : 0;
        d.pre = partials_[pre[k]];
        d.dmat = mat(dmat[k]);
        d.dmatt = mat_t(dmat[k]);
        d.dpad = mat_pad_[dmat[k]];
        d.reserved = 0;
    }
    return kSuccess;
}

int Instance::calculateEdgeDerivatives(const int* post, const int* pre, const int* dmat,
                                       const int* cw, int count, double* outDerivs,
                                       double* outSum, double* outSumSq) {
    const int rc = queue_edge_derivatives(post, pre, dmat, cw, count, outDerivs != nullptr);
    if (rc || count == 0) return rc;
    return deliver_sums(count, outDerivs, outSum, outSumSq);
}

// The launches of calculateEdgeDerivatives: the 2 * count sums into out_ and,
// with `site`, the per-site values into site_d_; nothing is delivered.
int Instance::queue_edge_derivatives(const int* post, const int* pre, const int* dmat,
                                     const int* cw, int count, bool site_values) {
    std::vector<DerivDesc> tab;
    const int rc0 = build_deriv(post, pre, dmat, cw, count, tab);
    if (rc0) return rc0;
    if (count == 0) return kSuccess;
    const int w = cw[0];
    const int nblk_generic = Pp_ / generic_tile_patterns(Sg_, dbl_);
    const int nblk_tc = Pp_ / tc_tile_patterns();
    const int nblk = S_ == 4 ? deriv_blocks(dims()) : std::max(nblk_generic, nblk_tc);
    CK(t_deriv_.upload(tab.data(), sizeof(DerivDesc) * count, stream_));
    CK(scratch_.reserve(sizeof(double) * 2 * (size_t)count * nblk));
    CK(out_.reserve(sizeof(double) * 2 * count));
    if (site_values) CK(site_d_.reserve(sizeof(double) * (size_t)count * P_));
    if (S_ == 4) {
        const DerivDesc* d_desc = (const DerivDesc*)t_deriv_.ptr;
        const double* catw = d_catw_ + (size_t)w * C_;
        double* site = site_values ? (double*)site_d_.ptr : nullptr;
        const Dims dm = dims();
        auto run = [&](int v) -> cudaError_t {
            return LAUNCH(launch_edge_derivatives, d_desc, count, catw, d_patw_, dm, site,
                          (double*)scratch_.ptr, (double*)out_.ptr, stream_, v);
        };
        const TuneKey key{kTuneDeriv, (int)dbl_, C_, Pp_, tune_count_class(count), device_};
        bulk_used_ = true;   // variant 6 may run (chosen, forced or being timed)
        const int v = tune_pick(key, deriv4_variants(dm), true, stream_, run);
        picked_[kTuneDeriv] = v;
        CK(run(v));
    } else {
        const DerivDesc* d_desc = (const DerivDesc*)t_deriv_.ptr;
        const double* catw = d_catw_ + (size_t)w * C_;
        double* site = site_values ? (double*)site_d_.ptr : nullptr;
        const Dims dm = dims();
        // variant 0: CUDA-core cluster kernel; 1: tensor cores (FP32 only)
        auto run = [&](int v) -> cudaError_t {
            cudaError_t e;
            if (v == 1) {
                tc_used_ = true;
                e = launch_deriv_tc(d_desc, count, catw, d_patw_, dm, site,
                                    (double*)scratch_.ptr, stream_);
            } else {
                e = LAUNCH(launch_deriv_generic, d_desc, count, catw, d_patw_, dm, site,
                           (double*)scratch_.ptr, stream_);
            }
            if (e != cudaSuccess) return e;
            return launch_deriv_final((double*)scratch_.ptr, v == 1 ? nblk_tc : nblk_generic,
                                      count, (double*)out_.ptr, stream_);
        };
        const bool tc = !dbl_ && tc_supported(dm);
        const TuneKey key{kTuneDeriv, (int)dbl_, C_ * 100 + Sg_, Pp_, tune_count_class(count),
                          device_};
        int v = tune_pick(key, tc ? 2 : 1, true, stream_, run);
        if (v < 0) v = tc ? 1 : 0;
        picked_[kTuneDeriv] = v;
        cudaError_t e = run(v);
        if (e == cudaErrorInvalidConfiguration && v == 1) {
            (void)cudaGetLastError();
            e = run(0);
        }
        CK(e);
    }
    return kSuccess;
}

// The 2 * count sums of an edge-derivative launch (out_), and the per-site
// values (site_d_) when requested, to the caller's arrays.
int Instance::deliver_sums(int count, double* outDerivs, double* outSum, double* outSumSq) {
    if (async_ && !outDerivs) {
        // ASYNCH: sums are written to the caller's arrays at the next
        // synchronisation point (getters, waitForPartials, synchronous calls).
        double* slot = stage(2 * (size_t)count);
        if (!slot) return kErrOOM;
        CK(cudaMemcpyAsync(slot, out_.ptr, sizeof(double) * 2 * count, cudaMemcpyDeviceToHost,
                           stream_));
        defer(Pending{slot, outSum, outSumSq, count});
        return kSuccess;
    }
    if ((size_t)2 * count > h_out_n_) {
        cudaFreeHost(h_out_);
        h_out_ = nullptr;
        h_out_n_ = 2 * count;
        CK(cudaMallocHost(&h_out_, sizeof(double) * h_out_n_));
    }
    CK(cudaMemcpyAsync(h_out_, out_.ptr, sizeof(double) * 2 * count, cudaMemcpyDeviceToHost,
                       stream_));
    if (outDerivs)
        CK(cudaMemcpyAsync(outDerivs, site_d_.ptr, sizeof(double) * (size_t)count * P_,
                           cudaMemcpyDeviceToHost, stream_));
    int rc = sync();
    if (rc) return rc;
    if (outSum) std::copy(h_out_, h_out_ + count, outSum);
    if (outSumSq) std::copy(h_out_ + count, h_out_ + 2 * count, outSumSq);
    return kSuccess;
}

// updatePrePartials(ops) then calculateEdgeDerivatives(post[k], dest of op k,
// dmat[k]) in one S = 4 walk (k_fused.cu) where the list allows it: at most
// 256 ops, no op rewriting a buffer that an earlier op's derivative reads (a
// destination written twice, or a post-order operand that is also a
// destination).  Otherwise the two calls run as they are; where the fused
// walk can run, the autotuner picks it or the two calls' kernels by time.
// Resolve the fused call's list: the pre-order walk table `tab`, the
// derivative table `dtab` and, for S = 4, the fused op list `fops` with its
// sibling-pair marks.  Returns kSuccess, kNotFused when only the two
// separate calls can run the list (no fused kernel for this shape, an op
// rewriting a buffer that an earlier op's derivative reads: a destination
// written twice, or a post-order operand that is also a destination), or an
// error code.
int Instance::build_prederiv(const int* ops, int count, const int* post, const int* dmat,
                             const int* cw, std::vector<OpDesc>& tab,
                             std::vector<DerivDesc>& dtab, std::vector<PreDerivOp>& fops,
                             bool& idempotent) {
    if (count < 0 || (count > 0 && (!ops || !post || !dmat || !cw))) return kErrRange;
    const Dims dm = dims();
    const bool tc_fused = !dbl_ && tc_supported(dm);
    if (count == 0 || !(fused_supported(dm, count) || tc_fused)) return kNotFused;
    std::vector<int> pre(count);
    for (int k = 0; k < count; ++k) pre[k] = ops[(size_t)k * 7];
    std::vector<uint8_t> dep;
    bool has_op_cum = false;
    idempotent = false;
    int rc = build_walk(ops, count, 7, true, tab, dep, idempotent, has_op_cum);
    if (rc) return rc;
    rc = build_deriv(post, pre.data(), dmat, cw, count, dtab);
    if (rc) return rc;
    std::unordered_map<int, int> writes;
    for (int k = 0; k < count; ++k) ++writes[pre[k]];
    for (int k = 0; k < count; ++k)
        if (writes[pre[k]] != 1 || writes.count(post[k])) return kNotFused;
    fops.clear();
    // Sibling pairs: same parent, each op's sibling the other's node, and
    // neither op's destination read by the other.
    std::vector<uint8_t> first(count, 0);
    for (int k = 0; k + 1 < count; ++k) {
        const int* a = ops + (size_t)k * 7;
        const int* b = a + 7;
        const bool pair = a[3] == b[3] && a[5] == post[k + 1] && b[5] == post[k] &&
                          a[0] != b[0] && a[0] != b[3] && a[0] != b[5] && a[0] != post[k + 1] &&
                          b[0] != a[5] && b[0] != post[k];
        if (pair) first[k++] = 1;
    }
    if (S_ != 4) {
        // the tensor-core pair walk reads the marks from the op list
        for (int k = 0; k < count; ++k)
            if (first[k]) tab[k].kind |= kPairFirst;
        return kSuccess;
    }
    fops.resize(count);
    for (int k = 0; k < count; ++k) {
        const OpDesc& t = tab[k];
        const DerivDesc& d = dtab[k];
        PreDerivOp& f = fops[k];
        f.parent = t.x1;
        f.sib = t.x2;
        f.dest = t.dest;
        f.mnode = t.m1;
        f.msib = t.m2;
        f.post = d.post;
        f.dmat = d.dmat;
        f.scale_write = t.scale_write;
        f.pad_sib = t.pad2;
        f.dpad = d.dpad;
        f.kind = (t.kind & (kX2States | kM1Transposed)) | (d.post_is_states ? kPostStates : 0);
        f.reserved = 0;
    }
    for (int k = 0; k + 1 < count; ++k) {
        if (first[k]) {
            fops[k].kind |= kPairFirst;
            const PreDerivOp &fa = fops[k], &fb = fops[k + 1];
            if (fa.mnode == fb.msib && fa.msib == fb.mnode &&
                !((fa.kind | fb.kind) & kM1Transposed))
                fops[k].kind |= kPairMats;
            if (fa.dmat == fb.dmat && fa.dpad == fb.dpad) fops[k].kind |= kPairD;
            ++k;
        }
    }
    return kSuccess;
}

int Instance::updatePrePartialsWithDerivatives(const int* ops, int count, const int* post,
                                               const int* dmat, const int* cw, double* outSum,
                                               double* outSumSq) {
    if (count < 0 || (count > 0 && (!ops || !post || !dmat || !cw))) return kErrRange;
    std::vector<int> pre(count);
    for (int k = 0; k < count; ++k) pre[k] = ops[(size_t)k * 7];
    auto separate = [&]() -> int {
        int rc = updatePrePartials(ops, count, -1);
        if (rc) return rc;
        return calculateEdgeDerivatives(post, pre.data(), dmat, cw, count, nullptr, outSum,
                                        outSumSq);
    };
    std::vector<OpDesc> tab;
    std::vector<DerivDesc> dtab;
    std::vector<PreDerivOp> fops;
    bool idempotent = false;
    const int rc = build_prederiv(ops, count, post, dmat, cw, tab, dtab, fops, idempotent);
    if (rc == kNotFused) return separate();
    if (rc) return rc;
    const Dims dm = dims();
    if (S_ != 4) return prederiv_tc(ops, count, post, pre.data(), dmat, cw, tab, dtab,
                                    idempotent, outSum, outSumSq);
    const int w = cw[0];
    const int nblk = std::max(fused_blocks(dm), deriv_blocks(dm));
    CK(scratch_.reserve(sizeof(double) * 2 * (size_t)count * nblk));
    CK(out_.reserve(sizeof(double) * 2 * count));
    CK(t_deriv_.upload(dtab.data(), sizeof(DerivDesc) * count, stream_));
    const double* catw = d_catw_ + (size_t)w * C_;
    const int ls = (int)log_scalers_;
    // Every variant leaves the sums in out_.  0: the pre-order walk and the
    // derivative kernels of the two calls; 1: the fused walk; 2: its
    // pairs-only form with 2 patterns a thread (FP32 lists of sibling pairs);
    // 3: the fused walk with its matrices staged in shared memory.  The autotuner
    // times them when the list may run repeatedly (no op reads what a later
    // op writes); the first, untimed run also settles the two calls' own
    // autotuner choices.
    auto run = [&](int v) -> cudaError_t {
        if (v == 0) {
            if (post_or_pre(ops, count, 7, -1, true) != kSuccess) return cudaErrorUnknown;
            const TuneKey dk{kTuneDeriv, (int)dbl_, C_, Pp_, tune_count_class(count), device_};
            bulk_used_ = true;
            auto deriv = [&](int dv) -> cudaError_t {
                return LAUNCH(launch_edge_derivatives, (const DerivDesc*)t_deriv_.ptr, count,
                              catw, d_patw_, dm, nullptr, (double*)scratch_.ptr,
                              (double*)out_.ptr, stream_, dv);
            };
            const int dv = tune_pick(dk, deriv4_variants(dm), true, stream_, deriv);
            picked_[kTuneDeriv] = dv;
            return deriv(dv);
        }
        return LAUNCH(launch_pre_deriv4, fops.data(), count, dm, catw, d_patw_, ls,
                      (double*)scratch_.ptr, (double*)out_.ptr, stream_, v);
    };
    const TuneKey key{kTuneFused, (int)dbl_, C_, Pp_, tune_count_class(count), device_};
    int v = tune_pick(key, 4, idempotent, stream_, run);
    if (v < 0) v = 1;
    cudaError_t e = run(v);
    if (e == cudaErrorInvalidValue && v == 2) {   // a forced pairs-only form the list refuses
        (void)cudaGetLastError();
        v = 1;
        e = run(v);
    }
    picked_[kTuneFused] = v;
    CK(e);
    return deliver_sums(count, nullptr, outSum, outSumSq);
}

// updatePrePartialsWithDerivatives for 4 < S <= 64 on the FP32 path.
// Variant 0: the two calls' kernels (each tuned as its own call); 1: the
// tensor-core fused walk (k_tc.cu k_prederiv_tc); 2: its sibling-pair form
// (k_prederiv_tc_pairs: 17 to 32 padded states, lists made only of sibling
// pairs; other lists run variant 1).  The autotuner times them when the list
// may run repeatedly.
int Instance::prederiv_tc(const int* ops, int count, const int* post, const int* pre,
                          const int* dmat, const int* cw, const std::vector<OpDesc>& tab,
                          const std::vector<DerivDesc>& dtab, bool idempotent, double* outSum,
                          double* outSumSq) {
    const Dims dm = dims();
    const int nblk = prederiv_tc_blocks(dm);
    CK(scratch_.reserve(sizeof(double) * 2 * (size_t)count * nblk));
    CK(out_.reserve(sizeof(double) * 2 * count));
    const double* catw = d_catw_ + (size_t)cw[0] * C_;
    const int ls = (int)log_scalers_;
    bool pairs_only = count % 2 == 0;          // every even op starts a sibling pair
    for (int k = 0; pairs_only && k < count; k += 2)
        pairs_only = (tab[k].kind & kPairFirst) != 0;
    auto run = [&](int v) -> cudaError_t {
        if (v == 0) {
            if (post_or_pre(ops, count, 7, -1, true) != kSuccess) return cudaErrorUnknown;
            if (queue_edge_derivatives(post, pre, dmat, cw, count, false) != kSuccess)
                return cudaErrorUnknown;
            return cudaSuccess;
        }
        if (v == 2 && !pairs_only) return cudaErrorInvalidValue;
        cudaError_t e = t_ops_pre_.upload(tab.data(), sizeof(OpDesc) * count, stream_);
        if (e == cudaSuccess) e = t_deriv_.upload(dtab.data(), sizeof(DerivDesc) * count, stream_);
        if (e != cudaSuccess) return e;
        tc_used_ = true;
        e = v == 2 ? launch_prederiv_tc_pairs((const OpDesc*)t_ops_pre_.ptr,
                                              (const DerivDesc*)t_deriv_.ptr, count, count, catw,
                                              d_patw_, dm, ls, (double*)scratch_.ptr, stream_)
                   : launch_prederiv_tc((const OpDesc*)t_ops_pre_.ptr,
                                        (const DerivDesc*)t_deriv_.ptr, count, count, catw,
                                        d_patw_, dm, ls, (double*)scratch_.ptr, stream_);
        if (e != cudaSuccess) return e;
        return launch_final_sum((double*)scratch_.ptr, nblk, 2 * count, (double*)out_.ptr,
                                stream_);
    };
    const TuneKey key{kTuneFused, (int)dbl_, C_ * 100 + Sg_, Pp_, tune_count_class(count),
                      device_};
    int v = tune_pick(key, 3, idempotent, stream_, run);
    if (v < 0) v = 1;
    cudaError_t e = run(v);
    if (e == cudaErrorInvalidValue && v == 2) {   // not a pairs-only list, or another width
        (void)cudaGetLastError();
        v = 1;
        e = run(v);
    }
    if (e == cudaErrorInvalidConfiguration && v >= 1) {   // TMEM could be oversubscribed
        (void)cudaGetLastError();
        v = 0;
        e = run(0);
    }
    picked_[kTuneFused] = v;
    CK(e);
    return deliver_sums(count, nullptr, outSum, outSumSq);
}

// beagleCalculateCrossProductDerivative (CPU/BeagleCPUImpl.hpp:1865-1937):
// the S x S sums over the listed branches are added into the caller's array
// (the reference adds, it does not clear); sums of squares are not written,
// as in the reference.  Synchronous.
int Instance::calculateCrossProducts(const int* post, const int* pre, const int* rates_idx,
                                     const int* cw, const double* lengths, int count,
                                     double* outSum) {
    if (count < 0 || (count > 0 && (!post || !pre || !rates_idx || !cw || !lengths)))
        return kErrRange;
    if (count == 0) return kSuccess;
    if (!outSum) return kErrRange;
    if (S_ > 64) return kErrNoImpl;
    const int ri = rates_idx[0], w = cw[0];
    if (ri < 0 || ri >= neig_ || !rates_set_[ri] || w < 0 || w >= neig_ || !catw_set_[w])
        return kErrRange;
    std::vector<DerivDesc> tab(count);
    std::vector<double> fac((size_t)count * C_);
    for (int k = 0; k < count; ++k) {
        if (!has_data(post[k]) || !buf_ok(pre[k]) || !partials_[pre[k]]) return kErrRange;
        DerivDesc& d = tab[k];
        d = DerivDesc{};
        d.post = states_[post[k]] ? (const void*)states_[post[k]] : partials_[post[k]];
        d.post_is_states = states_[post[k]] ? 1 : 0;
        d.pre = partials_[pre[k]];
        for (int c = 0; c < C_; ++c)
            fac[(size_t)k * C_ + c] =
                h_catw_[(size_t)w * C_ + c] * h_rates_[(size_t)ri * C_ + c] * lengths[k];
    }
    const Dims dm = dims();
    const int ntiles = (P_ + cross_tile_patterns(dm, dbl_) - 1) / cross_tile_patterns(dm, dbl_);
    const int SS = S_ * S_;
    CK(t_deriv_.upload(tab.data(), sizeof(DerivDesc) * count, stream_));
    CK(t_cross_.upload(fac.data(), sizeof(double) * fac.size(), stream_));
    CK(scratch_.reserve(sizeof(double) * (size_t)SS * ntiles));
    CK(out_.reserve(sizeof(double) * SS));
    CK(LAUNCH(launch_cross_products, (const DerivDesc*)t_deriv_.ptr, count,
              d_catw_ + (size_t)w * C_, (const double*)t_cross_.ptr, d_patw_, dm,
              (double*)scratch_.ptr, (double*)out_.ptr, stream_));
    std::vector<double> h(SS);
    CK(cudaMemcpyAsync(h.data(), out_.ptr, sizeof(double) * SS, cudaMemcpyDeviceToHost, stream_));
    const int rc = sync();
    if (rc) return rc;
    for (int q = 0; q < SS; ++q) outSum[q] += h[q];
    return kSuccess;
}

int Instance::calculateEdgeLogLikelihoods(const int* parents, const int* children,
                                          const int* prob, const int* d1, const int* d2,
                                          const int* cw, const int* sf, const int* cum, int count,
                                          double* outLnL, double* outD1, double* outD2) {
    if (count != 1) return kErrNoImpl;
    if (!parents || !children || !prob || !cw || !sf || !outLnL) return kErrRange;
    const int pa = parents[0], ch = children[0], pm = prob[0], w = cw[0], f = sf[0];
    const int c = cum ? cum[0] : -1;
    if (!buf_ok(pa) || !partials_[pa] || !has_data(ch)) return kErrRange;
    if (pm < 0 || pm >= nmat_) return kErrRange;
    const int m1 = d1 ? d1[0] : -1, m2 = (d1 && d2) ? d2[0] : -1;
    if ((d1 && (m1 < 0 || m1 >= nmat_)) || (m2 != -1 && (m2 < 0 || m2 >= nmat_)))
        return kErrRange;
    if (w < 0 || w >= neig_ || !catw_set_[w] || f < 0 || f >= neig_ || !freqs_set_[f])
        return kErrRange;
    if (c != -1 && (c < 0 || c >= nscale_)) return kErrRange;
    const int nblk = reduction_blocks(P_);
    CK(scratch_.reserve(sizeof(double) * 3 * nblk));
    CK(out_.reserve(sizeof(double) * 4));
    const bool st = states_[ch] != nullptr;
    CK(LAUNCH(launch_edge_lnl, partials_[pa], st ? (const void*)states_[ch] : partials_[ch],
              (int)st, mat(pm), mat_pad_[pm], m1 >= 0 ? mat(m1) : nullptr,
              m1 >= 0 ? mat_pad_[m1] : 0.0, m2 >= 0 ? mat(m2) : nullptr,
              m2 >= 0 ? mat_pad_[m2] : 0.0, d_catw_ + (size_t)w * C_, d_freqs_ + (size_t)f * S_,
              c >= 0 ? scale(c) : nullptr, d_patw_, dims(), d_site_, d_site1_, d_site2_,
              (double*)scratch_.ptr, (double*)out_.ptr, stream_));
    CK(cudaMemcpyAsync(h_out_, out_.ptr, sizeof(double) * 3, cudaMemcpyDeviceToHost, stream_));
    int rc = sync();
    if (rc) return rc;
    *outLnL = h_out_[0];
    last_lnl_ = h_out_[0];
    last_d1_ = h_out_[1];
    last_d2_ = h_out_[2];
    if (outD1 && m1 >= 0) *outD1 = h_out_[1];
    if (outD2 && m2 >= 0) *outD2 = h_out_[2];
    return std::isnan(*outLnL) ? kErrFP : kSuccess;
}

// CPU/BeagleCPUImpl.hpp:3008-3110 (count 1): per partition i the edge lnL of
// (parents[i], children[i], prob[i]) over partition parts[i]'s patterns, and
// their total; with both derivative matrices, the first and second derivative
// sums as well (:3452-3587).  A first derivative without a second is
// NO_IMPLEMENTATION there, and here.
int Instance::calculateEdgeLogLikelihoodsByPartition(
    const int* parents, const int* children, const int* prob, const int* d1, const int* d2,
    const int* cw, const int* sf, const int* cum, const int* parts, int nparts, int count,
    double* outByPart, double* out, double* outD1ByPart, double* outD1, double* outD2ByPart,
    double* outD2) {
    if (count != 1) return kErrNoImpl;
    if ((d1 != nullptr) != (d2 != nullptr)) return kErrNoImpl;
    const bool derivs = d1 != nullptr;
    if (nparts < 1 || !parents || !children || !prob || !cw || !sf || !parts || !outByPart ||
        !out)
        return kErrRange;
    if (derivs && (!outD1ByPart || !outD1 || !outD2ByPart || !outD2)) return kErrRange;
    if (partition_start_.empty()) return kErrRange;
    const int npart_defined = (int)partition_start_.size() - 1;
    int total_blocks = 0;
    for (int i = 0; i < nparts; ++i) {
        const int pa = parents[i], ch = children[i], pm = prob[i], w = cw[i], f = sf[i];
        const int c = cum ? cum[i] : -1, q = parts[i];
        if (!buf_ok(pa) || !partials_[pa] || !has_data(ch)) return kErrRange;
        if (pm < 0 || pm >= nmat_) return kErrRange;
        if (derivs && (d1[i] < 0 || d1[i] >= nmat_ || d2[i] < 0 || d2[i] >= nmat_))
            return kErrRange;
        if (w < 0 || w >= neig_ || !catw_set_[w] || f < 0 || f >= neig_ || !freqs_set_[f])
            return kErrRange;
        if (c != -1 && (c < 0 || c >= nscale_)) return kErrRange;
        if (q < 0 || q >= npart_defined) return kErrRange;
        total_blocks += 3 * reduction_blocks(partition_start_[q + 1] - partition_start_[q]);
    }
    CK(scratch_.reserve(sizeof(double) * std::max(total_blocks, 1)));
    CK(out_.reserve(sizeof(double) * 3 * nparts));
    double* blocks = (double*)scratch_.ptr;
    for (int i = 0; i < nparts; ++i) {
        const int pa = parents[i], ch = children[i], pm = prob[i], w = cw[i], f = sf[i];
        const int c = cum ? cum[i] : -1, q = parts[i];
        const int p0 = partition_start_[q], p1 = partition_start_[q + 1];
        const int m1 = derivs ? d1[i] : -1, m2 = derivs ? d2[i] : -1;
        const bool st = states_[ch] != nullptr;
        CK(LAUNCH(launch_edge_lnl_range, partials_[pa],
                  st ? (const void*)states_[ch] : partials_[ch], (int)st, mat(pm), mat_pad_[pm],
                  m1 >= 0 ? mat(m1) : nullptr, m1 >= 0 ? mat_pad_[m1] : 0.0,
                  m2 >= 0 ? mat(m2) : nullptr, m2 >= 0 ? mat_pad_[m2] : 0.0,
                  d_catw_ + (size_t)w * C_, d_freqs_ + (size_t)f * S_,
                  c >= 0 ? scale(c) : nullptr, d_patw_, dims(), p0, p1, d_site_, d_site1_,
                  d_site2_, blocks, (double*)out_.ptr + 3 * i, stream_));
        blocks += 3 * reduction_blocks(p1 - p0);
    }
    if ((size_t)(3 * nparts) > h_out_n_) {
        cudaFreeHost(h_out_);
        h_out_ = nullptr;
        h_out_n_ = 3 * nparts;
        CK(cudaMallocHost(&h_out_, sizeof(double) * h_out_n_));
    }
    CK(cudaMemcpyAsync(h_out_, out_.ptr, sizeof(double) * 3 * nparts, cudaMemcpyDeviceToHost,
                       stream_));
    int rc = sync();
    if (rc) return rc;
    double tot = 0, tot1 = 0, tot2 = 0;
    for (int i = 0; i < nparts; ++i) {
        outByPart[i] = h_out_[3 * i];
        tot += h_out_[3 * i];
        if (derivs) {
            outD1ByPart[i] = h_out_[3 * i + 1];
            outD2ByPart[i] = h_out_[3 * i + 2];
            tot1 += h_out_[3 * i + 1];
            tot2 += h_out_[3 * i + 2];
        }
    }
    *out = tot;
    last_lnl_ = tot;
    if (derivs) {
        *outD1 = tot1;
        *outD2 = tot2;
        last_d1_ = tot1;
        last_d2_ = tot2;
    }
    return (std::isnan(tot) || std::isnan(tot1) || std::isnan(tot2)) ? kErrFP : kSuccess;
}

int Instance::getLogLikelihood(double* out) {
    if (!out) return kErrRange;
    int rc = sync();
    if (rc) return rc;
    *out = last_lnl_;
    return std::isnan(last_lnl_) ? kErrFP : kSuccess;
}

int Instance::getDerivatives(double* d1, double* d2) {
    int rc = sync();
    if (rc) return rc;
    if (d1) *d1 = last_d1_;
    if (d2) *d2 = last_d2_;
    return kSuccess;
}

int Instance::getSiteLogLikelihoods(double* out) {
    if (!out) return kErrRange;
    CK(cudaMemcpyAsync(out, d_site_, sizeof(double) * P_, cudaMemcpyDeviceToHost, stream_));
    return sync();
}

int Instance::getSiteDerivatives(double* d1, double* d2) {
    if (d1) CK(cudaMemcpyAsync(d1, d_site1_, sizeof(double) * P_, cudaMemcpyDeviceToHost, stream_));
    if (d2) CK(cudaMemcpyAsync(d2, d_site2_, sizeof(double) * P_, cudaMemcpyDeviceToHost, stream_));
    return sync();
}

}  // namespace b200
