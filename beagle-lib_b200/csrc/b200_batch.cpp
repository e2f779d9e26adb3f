// Batched calls over several instances; see b200_batch.h.
#include "b200_batch.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>

namespace b200 {

namespace {

enum { kSuccess = 0, kErrGeneral = -1, kErrOOM = -2, kErrRange = -5, kErrFP = -8 };

#define CK(call)                                                              \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) {                                              \
            (void)cudaGetLastError();                                         \
            return e_ == cudaErrorMemoryAllocation ? kErrOOM : kErrGeneral;   \
        }                                                                     \
    } while (0)

#define LAUNCH(fn, ...) (dbl_ ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

// 4-state members with a lane-group category count run in the batched kernels.
bool batched4(const Instance* in, int S, int C) {
    (void)in;
    return S == 4 && (C == 1 || C == 2 || C == 4 || C == 8);
}

int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Bytes of `v`, appended to a byte table at a 256-byte aligned offset.
template <typename T>
size_t append(std::vector<unsigned char>& table, const std::vector<T>& v) {
    const size_t off = (table.size() + 255) & ~size_t(255);
    table.resize(off + sizeof(T) * v.size());
    if (!v.empty()) std::memcpy(table.data() + off, v.data(), sizeof(T) * v.size());
    return off;
}

}  // namespace

Batch::~Batch() {
    release();
    for (GraphRec& g : graphs_) free_graph(g);
    for (DevBuf* b : {&t_a_, &t_b_, &t_c_, &t_block_, &t_out_, &t_out2_}) b->release();
    for (auto& c : chunks_) cudaFreeHost(c.first);
    if (fork_ev_) cudaEventDestroy(fork_ev_);
    if (join_ev_) cudaEventDestroy(join_ev_);
    if (side_) cudaStreamDestroy(side_);
    if (stream_) cudaStreamDestroy(stream_);
}

cudaError_t Batch::fork() {
    cudaError_t e = cudaEventRecord(fork_ev_, stream_);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side_, fork_ev_, 0);
    return e;
}

cudaError_t Batch::join() {
    cudaError_t e = cudaEventRecord(join_ev_, side_);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream_, join_ev_, 0);
    return e;
}

int Batch::create(const std::vector<Instance*>& members) {
    if (members.empty()) return kErrRange;
    device_ = members[0]->device_;
    dbl_ = members[0]->dbl_;
    for (Instance* in : members)
        if (!in || in->device_ != device_ || in->dbl_ != dbl_) return kErrRange;
    for (size_t i = 0; i < members.size(); ++i)
        for (size_t j = i + 1; j < members.size(); ++j)
            if (members[i] == members[j]) return kErrRange;
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&join_ev_, cudaEventDisableTiming));
    for (Instance* in : members) {
        const int rc = in->use_stream(stream_);
        if (rc) return rc;
        m_.push_back(in);
    }
    return kSuccess;
}

void Batch::release() {
    if (capturing_) {   // an unfinished capture is dropped
        int g = -1;
        (void)endCapture(&g);
        if (g >= 0) free_graph(graphs_[g]);
    }
    if (!m_.empty()) wait();
    for (Instance* in : m_) in->use_stream(nullptr);
    m_.clear();
}

bool Batch::deferred() const {
    for (const Instance* in : m_)
        if (!in->async_) return false;
    return true;
}

int Batch::sync() {
    if (capturing_) return kErrGeneral;   // a wait would break the capture
    CK(cudaStreamSynchronize(stream_));
    for (const Pending& pd : pending_) {
        std::copy(pd.src, pd.src + pd.n, pd.dst);
        if (pd.member >= 0) m_[pd.member]->last_lnl_ = pd.src[0];
    }
    pending_.clear();
    chunk_i_ = 0;
    chunk_off_ = 0;
    // Members that ran their own result calls (ASYNCH) deliver theirs too.
    for (Instance* in : m_)
        if (!in->pending_.empty()) {
            const int rc = in->sync();
            if (rc) return rc;
        }
    return kSuccess;
}

int Batch::wait() { return sync(); }

void Batch::push_pending(const Pending& pd) {
    if (capturing_) cap_.deliveries.push_back(pd);
    else pending_.push_back(pd);
}

// n doubles of pinned staging, valid until the next sync(); while capturing,
// a block the graph owns (its copy writes there at every launch).
double* Batch::stage(size_t n) {
    if (capturing_) {
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
        const size_t sz = std::max<size_t>(n, 1 << 16);
        double* p = nullptr;
        if (cudaMallocHost(&p, sizeof(double) * sz) != cudaSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        chunks_.emplace_back(p, sz);
    }
    double* p = chunks_[chunk_i_].first + chunk_off_;
    chunk_off_ += n;
    return p;
}

// ------------------------------------------------------------ CUDA graphs
// The batch's calls between beginCapture and endCapture become one CUDA graph
// of the shared stream: the batched kernels, the members' own launches, every
// table upload (through pinned blocks the graph owns) and every result copy.
// Members are marked as capturing, so their own result copies and deliveries
// are recorded too and no call may wait.  Results of a launch are delivered at
// the next wait(), as the captured calls' would be.  The captured sequence
// must have run once before (its tables and scratch are then sized).
int Batch::beginCapture() {
    if (capturing_ || !deferred()) return kErrGeneral;
    for (Instance* in : m_)
        if (in->capturing_) return kErrGeneral;
    int rc = sync();
    if (rc) return rc;
    cap_ = GraphRec{};
    // room for the captured matrix updates' branch lengths (allocated before
    // the capture starts: the graph keeps the address)
    for (Instance* in : m_) cap_.len_cap += 4 * in->nmat_;
    CK(cudaMalloc(&cap_.d_len, sizeof(double) * std::max(cap_.len_cap, 1)));
    const cudaError_t e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        free_graph(cap_);
        return kErrGeneral;
    }
    capturing_ = true;
    capture_pinned() = &cap_.pinned;
    for (Instance* in : m_) {
        in->cap_ = Instance::GraphRec{};
        in->capturing_ = true;
    }
    return kSuccess;
}

int Batch::endCapture(int* graph) {
    if (!capturing_ || !graph) return kErrGeneral;
    capturing_ = false;
    capture_pinned() = nullptr;
    for (size_t i = 0; i < m_.size(); ++i) {
        Instance* in = m_[i];
        in->capturing_ = false;
        if (!in->cap_.deliveries.empty())
            cap_.member_deliveries.emplace_back((int)i, std::move(in->cap_.deliveries));
        cap_.pinned.insert(cap_.pinned.end(), in->cap_.pinned.begin(), in->cap_.pinned.end());
        in->cap_ = Instance::GraphRec{};
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&cap_.exec, g, 0ULL);
    cap_.graph = g;
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        free_graph(cap_);
        return kErrGeneral;
    }
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
    graphs_.push_back(std::move(cap_));
    cap_ = GraphRec{};
    *graph = (int)graphs_.size() - 1;
    return kSuccess;
}

// The lengths are copied on the host into one of the graph's pinned slots
// before this call returns; the slot's copy to the device is stream-ordered
// before the launch, and a slot is rewritten only after its last copy ran.
int Batch::launchGraphWithLengths(int graph, const double* lengths, int count) {
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

int Batch::launchGraph(int graph) {
    if (capturing_ || graph < 0 || graph >= (int)graphs_.size() || !graphs_[graph].exec)
        return kErrRange;
    note_graph_launch();
    CK(cudaGraphLaunch(graphs_[graph].exec, stream_));
    const GraphRec& g = graphs_[graph];
    for (const Pending& pd : g.deliveries) pending_.push_back(pd);
    for (const auto& md : g.member_deliveries)
        for (const Instance::Pending& pd : md.second) m_[md.first]->pending_.push_back(pd);
    return kSuccess;
}

void Batch::free_graph(GraphRec& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    for (void* p : g.pinned) cudaFreeHost(p);
    if (g.d_len) cudaFree(g.d_len);
    for (cudaEvent_t ev : g.len_ev)
        if (ev) cudaEventDestroy(ev);
    if (g.h_len_ring) cudaFreeHost(g.h_len_ring);
    g = GraphRec{};
}

// ------------------------------------------------------------ matrices
int Batch::updateTransitionMatrices(const int* eig, const int* const* prob,
                                    const double* const* t, const int* counts) {
    const int n = size();
    std::map<std::tuple<int, int, int>, std::vector<MatJob>> groups;   // (S, Sg, C) -> jobs
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        std::vector<MatJob> jobs;
        std::vector<int> e(std::max(counts[i], 0), eig ? eig[i] : 0), r(e.size(), 0);
        const int rc = in->build_matrix_jobs(e.data(), r.data(), prob[i], nullptr, nullptr, t[i],
                                             counts[i], jobs);
        if (rc) return rc;
        if (capturing_ && cap_.d_len) {
            // the graph reads these lengths from d_len (launchGraphWithLengths)
            if ((int)(cap_.len.size() + jobs.size()) > cap_.len_cap) {
                cap_.len_all = false;
            } else {
                for (MatJob& j : jobs) {
                    j.tlen = cap_.d_len + cap_.len.size();
                    cap_.len.push_back(j.t);
                }
            }
        }
        auto& g = groups[std::make_tuple(in->S_, in->Sg_, in->C_)];
        g.insert(g.end(), jobs.begin(), jobs.end());
    }
    std::vector<unsigned char> table;
    std::vector<std::pair<size_t, size_t>> where;   // (offset, jobs) per group
    for (auto& kv : groups) where.emplace_back(append(table, kv.second), kv.second.size());
    if (table.empty()) return kSuccess;
    CK(t_a_.upload(table.data(), table.size(), stream_));
    size_t k = 0;
    for (auto& kv : groups) {
        const Dims d{std::get<0>(kv.first), std::get<1>(kv.first), 0, 0, std::get<2>(kv.first)};
        const MatJob* jobs = (const MatJob*)((unsigned char*)t_a_.ptr + where[k].first);
        CK(LAUNCH(launch_update_matrices, jobs, (int)where[k].second, d, stream_));
        ++k;
    }
    return kSuccess;
}

// ----------------------------------------------------------------- walks
int Batch::updatePartials(const int* const* ops, const int* counts, const int* cumulative,
                          bool pre) {
    const int n = size();
    struct Member {
        int i;
        size_t ops_off;
        int nops;
    };
    std::map<int, std::vector<Member>> groups;   // C -> batched 4-state members
    // (S, Sg, C) -> FP32 members of the batched tensor-core walk
    std::map<std::tuple<int, int, int>, std::vector<Member>> tcgroups;
    std::vector<unsigned char> table;
    std::vector<int> fallback;
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        const int cum = cumulative ? cumulative[i] : -1;
        if (cum != -1 && (cum < 0 || cum >= in->nscale_)) return kErrRange;
        if (!batched4(in, in->S_, in->C_)) {
            if (!dbl_ && tc_supported(in->dims())) {
                std::vector<OpDesc> tab;
                std::vector<uint8_t> dep;
                bool idem = true, has_cum = false;
                const int rc = in->build_walk(ops[i], counts[i], 7, pre, tab, dep, idem, has_cum);
                if (rc) return rc;
                if (tab.empty()) continue;
                tcgroups[std::make_tuple(in->S_, in->Sg_, in->C_)].push_back(
                    Member{i, append(table, tab), (int)tab.size()});
                continue;
            }
            fallback.push_back(i);
            continue;
        }
        std::vector<OpDesc> tab;
        std::vector<uint8_t> dep;
        bool idem = true, has_cum = false;
        const int rc = in->build_walk(ops[i], counts[i], 7, pre, tab, dep, idem, has_cum);
        if (rc) return rc;
        if (tab.empty()) continue;
        groups[in->C_].push_back(Member{i, append(table, tab), (int)tab.size()});
    }
    // Single-instance launches of the other members (shared stream).
    for (int i : fallback) {
        const int rc = m_[i]->post_or_pre(ops[i], counts[i], 7, cumulative ? cumulative[i] : -1,
                                          pre);
        if (rc) return rc;
    }
    if (groups.empty() && tcgroups.empty()) return kSuccess;
    CK(t_a_.upload(table.data(), table.size(), stream_));
    // Segment tables (device pointers into t_a_), one per category count.
    std::vector<unsigned char> segtab;
    struct G {
        int C;
        size_t off;
        int nseg;
        int ncta;
    };
    std::vector<G> gl;
    struct TG {
        Dims d;
        size_t off;
        int nseg;
        int ntiles;
        std::vector<int> members;
    };
    std::vector<TG> tgl;
    for (auto& kv : tcgroups) {
        std::vector<WalkSeg> segs;
        TG tg{};
        tg.d = Dims{std::get<0>(kv.first), std::get<1>(kv.first), 0, 0, std::get<2>(kv.first)};
        for (const Member& mb : kv.second) {
            Instance* in = m_[mb.i];
            const int cum = cumulative ? cumulative[mb.i] : -1;
            WalkSeg sg{};
            sg.ops = (const OpDesc*)((unsigned char*)t_a_.ptr + mb.ops_off);
            sg.cum = (!pre && cum >= 0) ? in->scale(cum) : nullptr;
            sg.nops = mb.nops;
            sg.Pp = in->Pp_;
            sg.log_scalers = (int)in->log_scalers_;
            sg.first_cta = tg.ntiles;                  // counted in 128-pattern tiles
            tg.ntiles += in->Pp_ / tc_tile_patterns();
            segs.push_back(sg);
            tg.members.push_back(mb.i);
        }
        tg.off = append(segtab, segs);
        tg.nseg = (int)segs.size();
        tgl.push_back(tg);
    }
    for (auto& kv : groups) {
        const int C = kv.first;
        std::vector<WalkSeg> segs;
        int cta = 0;
        for (const Member& mb : kv.second) {
            Instance* in = m_[mb.i];
            const int cum = cumulative ? cumulative[mb.i] : -1;
            WalkSeg sg{};
            sg.ops = (const OpDesc*)((unsigned char*)t_a_.ptr + mb.ops_off);
            sg.cum = (!pre && cum >= 0) ? in->scale(cum) : nullptr;
            sg.nops = mb.nops;
            sg.Pp = in->Pp_;
            sg.log_scalers = (int)in->log_scalers_;
            sg.first_cta = cta;
            cta += ceil_div(in->Pp_, 256 / C);
            segs.push_back(sg);
        }
        gl.push_back(G{C, append(segtab, segs), (int)segs.size(), cta});
    }
    CK(t_b_.upload(segtab.data(), segtab.size(), stream_));
    // the tensor-core groups on the second stream, beside the 4-state ones
    const bool split = !gl.empty() && !tgl.empty();
    if (split) CK(fork());
    cudaError_t err = cudaSuccess;
    std::vector<const TG*> late;   // tensor-core shapes that cannot launch here
    for (const TG& g : tgl) {
        const cudaError_t e = launch_walk_tc_batch(
            (const WalkSeg*)((unsigned char*)t_b_.ptr + g.off), g.nseg, g.ntiles, pre, g.d,
            split ? side_ : stream_);
        if (e == cudaErrorInvalidConfiguration) {
            (void)cudaGetLastError();
            late.push_back(&g);
            continue;
        }
        if (e != cudaSuccess) err = e;
        for (int i : g.members) m_[i]->tc_used_ = true;
    }
    for (const G& g : gl) {
        if (err != cudaSuccess) break;
        err = LAUNCH(launch_walk4_batch, (const WalkSeg*)((unsigned char*)t_b_.ptr + g.off),
                     g.nseg, g.ncta, g.C, pre, stream_);
    }
    if (split) {
        const cudaError_t e = join();
        if (err == cudaSuccess) err = e;
    }
    CK(err);
    for (const TG* g : late)   // the members' own walks
        for (int i : g->members) {
            const int rc = m_[i]->post_or_pre(ops[i], counts[i], 7,
                                              cumulative ? cumulative[i] : -1, pre);
            if (rc) return rc;
        }
    return kSuccess;
}

// ---------------------------------------------------------- scale factors
int Batch::accumulateScaleFactors(const int* const* idx, const int* counts,
                                  const int* cumulative, int reset) {
    const int n = size();
    std::vector<unsigned char> itab;
    std::vector<size_t> ioff(n);
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        if (cumulative[i] < 0 || cumulative[i] >= in->nscale_ || counts[i] < 0) return kErrRange;
        std::vector<int> v(idx[i], idx[i] + counts[i]);
        for (int x : v)
            if (x < 0 || x >= in->nscale_) return kErrRange;
        ioff[i] = append(itab, v);
    }
    if (itab.empty()) itab.resize(16);
    CK(t_a_.upload(itab.data(), itab.size(), stream_));
    std::vector<AccSeg> segs(n);
    int cta = 0;
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        AccSeg& sg = segs[i];
        sg.cum = in->scale(cumulative[i]);
        sg.pool = in->d_scale_;
        sg.idx = (const int*)((unsigned char*)t_a_.ptr + ioff[i]);
        sg.n = counts[i];
        sg.Pp = in->Pp_;
        sg.P = in->P_;
        sg.log_scalers = (int)in->log_scalers_;
        sg.reset = reset;
        sg.first_cta = cta;
        cta += ceil_div(in->P_, accumulate_batch_patterns());
    }
    CK(t_b_.upload(segs.data(), sizeof(AccSeg) * n, stream_));
    CK(launch_accumulate_batch((const AccSeg*)t_b_.ptr, n, cta, stream_));
    return kSuccess;
}

// --------------------------------------------------------- root partials
int Batch::setRootPrePartials(const int* bufs, const int* freqs) {
    const int n = size();
    std::vector<FillSeg> segs(n);
    int cta = 0;
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        const int b = bufs[i], f = freqs[i];
        if (!in->buf_ok(b) || f < 0 || f >= in->neig_ || !in->freqs_set_[f]) return kErrRange;
        const int rc = in->ensure_partials(b);
        if (rc) return rc;
        FillSeg& sg = segs[i];
        sg.dest = in->partials_[b];
        sg.freqs = in->d_freqs_ + (size_t)f * in->S_;
        sg.n = (long long)in->Pp_ * in->C_ * in->Sg_;
        sg.S = in->S_;
        sg.Sg = in->Sg_;
        sg.first_cta = cta;
        cta += ceil_div(sg.n, 256);
    }
    CK(t_c_.upload(segs.data(), sizeof(FillSeg) * n, stream_));
    CK(LAUNCH(launch_fill_batch, (const FillSeg*)t_c_.ptr, n, cta, stream_));
    return kSuccess;
}

// ----------------------------------------------------------- root lnL
int Batch::rootLogLikelihoods(const int* bufs, const int* cw, const int* sf, const int* cum,
                              double* out) {
    const int n = size();
    std::vector<RootSeg> segs(n);
    std::vector<FinalSeg> fin(n);
    int cta = 0;
    size_t blocks = 0;
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        const int b = bufs[i], w = cw[i], f = sf[i], c = cum ? cum[i] : -1;
        if (!in->buf_ok(b) || !in->partials_[b]) return kErrRange;
        if (w < 0 || w >= in->neig_ || !in->catw_set_[w] || f < 0 || f >= in->neig_ ||
            !in->freqs_set_[f])
            return kErrRange;
        if (c != -1 && (c < 0 || c >= in->nscale_)) return kErrRange;
        const int nblk = reduction_blocks(in->P_);
        RootSeg& sg = segs[i];
        sg.root = in->partials_[b];
        sg.catw = in->d_catw_ + (size_t)w * in->C_;
        sg.freqs = in->d_freqs_ + (size_t)f * in->S_;
        sg.cum = c >= 0 ? in->scale(c) : nullptr;
        sg.patw = in->d_patw_;
        sg.site = in->d_site_;
        sg.block = nullptr;   // set below, after t_block_ is sized
        sg.S = in->S_;
        sg.Sg = in->Sg_;
        sg.C = in->C_;
        sg.P = in->P_;
        sg.first_cta = cta;
        cta += nblk;
        fin[i].nblk = nblk;
        fin[i].nout = 1;
        fin[i].first_out = i;
        blocks += nblk;
    }
    CK(t_block_.reserve(sizeof(double) * std::max<size_t>(blocks, 1)));
    CK(t_out_.reserve(sizeof(double) * n));
    size_t boff = 0;
    for (int i = 0; i < n; ++i) {
        segs[i].block = (double*)t_block_.ptr + boff;
        fin[i].block = segs[i].block;
        fin[i].out = (double*)t_out_.ptr + i;
        boff += fin[i].nblk;
    }
    std::vector<unsigned char> table;
    const size_t o1 = append(table, segs), o2 = append(table, fin);
    CK(t_c_.upload(table.data(), table.size(), stream_));
    CK(LAUNCH(launch_root_batch, (const RootSeg*)((unsigned char*)t_c_.ptr + o1), n, cta,
              stream_));
    CK(launch_final_batch((const FinalSeg*)((unsigned char*)t_c_.ptr + o2), n, n, stream_));
    double* h = stage(n);
    if (!h) return kErrOOM;
    CK(cudaMemcpyAsync(h, t_out_.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_));
    for (int i = 0; i < n; ++i) push_pending(Pending{h + i, out + i, 1, i});
    if (deferred()) return kSuccess;   // delivered by wait()
    int rc = sync();
    if (rc) return rc;
    bool nan = false;
    for (int i = 0; i < n; ++i) nan = nan || std::isnan(out[i]);
    return nan ? kErrFP : kSuccess;
}

// ---------------------------------- post-order walk + scaling + root lnL
// Per member, updatePartialsWithRootLogLikelihood (Instance:: semantics):
// updatePartials(ops, NONE); with a cumulative buffer, resetScaleFactors on
// it and accumulateScaleFactors of the list's scale buffers; then the root
// lnL.  When every member is a 4-state one with 1, 2, 4 or 8 categories, a
// list of at least one op ending at its root and not rewriting its
// cumulative buffer: one k_post4root_batch launch per category count, one
// final sum for all.  Otherwise the batched calls of the three steps.
int Batch::postRoot(const int* const* ops, const int* counts, const int* cumulative,
                    const int* roots, const int* cw, const int* sf, double* out) {
    const int n = size();
    bool fused = true;
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        const int cum = cumulative[i];
        if (counts[i] < 0 || (counts[i] > 0 && !ops[i])) return kErrRange;
        if (cum != -1 && (cum < 0 || cum >= in->nscale_)) return kErrRange;
        bool ok = batched4(in, in->S_, in->C_) && in->Sg_ == 4 && counts[i] >= 1 &&
                  ops[i][(size_t)(counts[i] - 1) * 7] == roots[i];
        for (int k = 0; ok && cum >= 0 && k < counts[i]; ++k)
            if (ops[i][(size_t)k * 7 + 1] == cum) ok = false;   // rewrites the cumulative buffer
        fused = fused && ok;
    }
    if (!fused) {
        std::vector<int> none(n, -1);
        int rc = updatePartials(ops, counts, none.data(), false);
        if (rc) return rc;
        std::vector<std::vector<int>> written(n);
        bool any = false, all = true;
        for (int i = 0; i < n; ++i) {
            any = any || cumulative[i] >= 0;
            all = all && cumulative[i] >= 0;
            for (int k = 0; k < counts[i]; ++k)
                if (ops[i][(size_t)k * 7 + 1] >= 0) written[i].push_back(ops[i][(size_t)k * 7 + 1]);
        }
        if (any && all) {
            std::vector<const int*> ip(n);
            std::vector<int> cnt(n);
            for (int i = 0; i < n; ++i) {
                ip[i] = written[i].data();
                cnt[i] = (int)written[i].size();
            }
            rc = accumulateScaleFactors(ip.data(), cnt.data(), cumulative, 1);
            if (rc) return rc;
        } else if (any) {
            for (int i = 0; i < n; ++i) {
                if (cumulative[i] < 0) continue;
                rc = m_[i]->resetScaleFactors(cumulative[i], -1);
                if (!rc)
                    rc = m_[i]->accumulateScaleFactors(written[i].data(), (int)written[i].size(),
                                                       cumulative[i], 1.0, -1);
                if (rc) return rc;
            }
        }
        return rootLogLikelihoods(roots, cw, sf, cumulative, out);
    }
    struct Member {
        int i;
        size_t off;
    };
    std::map<int, std::vector<Member>> groups;   // C -> members
    std::vector<unsigned char> table;
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        const int w = cw[i], f = sf[i];
        if (!in->buf_ok(roots[i]) || w < 0 || w >= in->neig_ || !in->catw_set_[w] || f < 0 ||
            f >= in->neig_ || !in->freqs_set_[f])
            return kErrRange;
        std::vector<OpDesc> tab;
        std::vector<uint8_t> dep;
        bool idem = true, has_cum = false;
        const int rc = in->build_walk(ops[i], counts[i], 7, false, tab, dep, idem, has_cum);
        if (rc) return rc;
        groups[in->C_].push_back(Member{i, append(table, tab)});
    }
    CK(t_a_.upload(table.data(), table.size(), stream_));
    size_t blocks = 0;
    for (int i = 0; i < n; ++i) blocks += (size_t)post_root_blocks(m_[i]->dims());
    CK(t_block_.reserve(sizeof(double) * std::max<size_t>(blocks, 1)));
    CK(t_out_.reserve(sizeof(double) * n));
    struct G {
        int C;
        size_t off;
        int nseg;
        int ncta;
    };
    std::vector<G> gl;
    std::vector<unsigned char> segtab;
    std::vector<FinalSeg> fin(n);
    size_t boff = 0;
    for (auto& kv : groups) {
        const int C = kv.first;
        std::vector<PostRootSeg> segs;
        int cta = 0;
        for (const Member& mb : kv.second) {
            Instance* in = m_[mb.i];
            PostRootSeg sg{};
            sg.ops = (const OpDesc*)((unsigned char*)t_a_.ptr + mb.off);
            sg.cum = cumulative[mb.i] >= 0 ? in->scale(cumulative[mb.i]) : nullptr;
            sg.catw = in->d_catw_ + (size_t)cw[mb.i] * in->C_;
            sg.freqs = in->d_freqs_ + (size_t)sf[mb.i] * in->S_;
            sg.patw = in->d_patw_;
            sg.site = in->d_site_;
            sg.block = (double*)t_block_.ptr + boff;
            sg.nops = counts[mb.i];
            sg.Pp = in->Pp_;
            sg.P = in->P_;
            sg.log_scalers = (int)in->log_scalers_;
            sg.first_cta = cta;
            cta += ceil_div(in->Pp_, post_root_batch_patterns(C));
            segs.push_back(sg);
            FinalSeg& f = fin[mb.i];
            f.block = sg.block;
            f.out = (double*)t_out_.ptr + mb.i;
            f.nblk = post_root_blocks(in->dims());
            f.nout = 1;
            f.first_out = mb.i;
            boff += (size_t)f.nblk;
        }
        gl.push_back(G{C, append(segtab, segs), (int)segs.size(), cta});
    }
    const size_t foff = append(segtab, fin);
    CK(t_b_.upload(segtab.data(), segtab.size(), stream_));
    for (const G& g : gl)
        CK(LAUNCH(launch_post4_root_batch, (const PostRootSeg*)((unsigned char*)t_b_.ptr + g.off),
                  g.nseg, g.ncta, g.C, stream_));
    CK(launch_final_batch((const FinalSeg*)((unsigned char*)t_b_.ptr + foff), n, n, stream_));
    double* h = stage(n);
    if (!h) return kErrOOM;
    CK(cudaMemcpyAsync(h, t_out_.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_));
    for (int i = 0; i < n; ++i) push_pending(Pending{h + i, out + i, 1, i});
    if (deferred()) return kSuccess;   // delivered by wait()
    int rc = sync();
    if (rc) return rc;
    bool nan = false;
    for (int i = 0; i < n; ++i) nan = nan || std::isnan(out[i]);
    return nan ? kErrFP : kSuccess;
}

// ------------------------------------------------------- edge derivatives
int Batch::edgeDerivatives(const int* const* post, const int* const* pre,
                           const int* const* dmat, const int* cw, const int* counts,
                           double* const* sums, double* const* sumsq) {
    const int n = size();
    struct Member {
        int i;
        size_t desc_off;
        int nb;
        int nblk;
    };
    std::map<int, std::vector<Member>> groups;
    std::map<std::tuple<int, int, int>, std::vector<Member>> tcgroups;   // (S, Sg, C), FP32
    std::vector<unsigned char> table;
    std::vector<int> fallback;
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        if (counts[i] <= 0) continue;
        const bool tc = !batched4(in, in->S_, in->C_) && !dbl_ && deriv_tc_launchable(in->dims());
        if (!batched4(in, in->S_, in->C_) && !tc) {
            fallback.push_back(i);
            continue;
        }
        std::vector<DerivDesc> tab;
        const int rc = in->build_deriv(post[i], pre[i], dmat[i], &cw[i], counts[i], tab);
        if (rc) return rc;
        if (tc)
            tcgroups[std::make_tuple(in->S_, in->Sg_, in->C_)].push_back(
                Member{i, append(table, tab), counts[i], in->Pp_ / tc_tile_patterns()});
        else
            groups[in->C_].push_back(Member{i, append(table, tab), counts[i],
                                            ceil_div(in->P_, deriv4_batch_tile(in->C_))});
    }
    for (int i : fallback) {
        const int rc = m_[i]->calculateEdgeDerivatives(post[i], pre[i], dmat[i], &cw[i],
                                                       counts[i], nullptr, sums[i], sumsq[i]);
        if (rc) return rc;
    }
    if (groups.empty() && tcgroups.empty()) return kSuccess;
    CK(t_a_.upload(table.data(), table.size(), stream_));
    size_t blocks = 0, outs = 0;
    for (auto& kv : groups)
        for (const Member& mb : kv.second) {
            blocks += (size_t)2 * mb.nb * mb.nblk;
            outs += (size_t)2 * mb.nb;
        }
    for (auto& kv : tcgroups)
        for (const Member& mb : kv.second) {
            blocks += (size_t)2 * mb.nb * mb.nblk;
            outs += (size_t)2 * mb.nb;
        }
    CK(t_block_.reserve(sizeof(double) * blocks));
    CK(t_out2_.reserve(sizeof(double) * outs));
    std::vector<unsigned char> segtab;
    struct G {
        int C;
        size_t off;
        int nseg;
        int ncta;
    };
    std::vector<G> gl;
    std::vector<FinalSeg> fin;
    std::vector<std::pair<int, size_t>> out_of;   // (member, first output) in t_out_
    size_t boff = 0, ooff = 0;
    for (auto& kv : groups) {
        std::vector<DerivSeg> segs;
        int cta = 0;
        for (const Member& mb : kv.second) {
            Instance* in = m_[mb.i];
            DerivSeg sg{};
            sg.desc = (const DerivDesc*)((unsigned char*)t_a_.ptr + mb.desc_off);
            sg.catw = in->d_catw_ + (size_t)cw[mb.i] * in->C_;
            sg.patw = in->d_patw_;
            sg.block = (double*)t_block_.ptr + boff;
            sg.nb = mb.nb;
            sg.P = in->P_;
            sg.nblk = mb.nblk;
            sg.first_cta = cta;
            cta += mb.nb * mb.nblk;
            segs.push_back(sg);
            FinalSeg f{};
            f.block = sg.block;
            f.out = (double*)t_out2_.ptr + ooff;
            f.nblk = mb.nblk;
            f.nout = 2 * mb.nb;
            f.first_out = (int)ooff;
            fin.push_back(f);
            out_of.emplace_back(mb.i, ooff);
            boff += (size_t)2 * mb.nb * mb.nblk;
            ooff += (size_t)2 * mb.nb;
        }
        gl.push_back(G{kv.first, append(segtab, segs), (int)segs.size(), cta});
    }
    // tensor-core groups: segment first_cta counts (branch, tile) clusters
    struct TG {
        Dims d;
        size_t off;
        int nseg;
        int nclusters;
        std::vector<int> members;
    };
    std::vector<TG> tgl;
    for (auto& kv : tcgroups) {
        std::vector<DerivSeg> segs;
        TG tg{};
        tg.d = Dims{std::get<0>(kv.first), std::get<1>(kv.first), 0, 0, std::get<2>(kv.first)};
        for (const Member& mb : kv.second) {
            Instance* in = m_[mb.i];
            DerivSeg sg{};
            sg.desc = (const DerivDesc*)((unsigned char*)t_a_.ptr + mb.desc_off);
            sg.catw = in->d_catw_ + (size_t)cw[mb.i] * in->C_;
            sg.patw = in->d_patw_;
            sg.block = (double*)t_block_.ptr + boff;
            sg.nb = mb.nb;
            sg.P = in->P_;
            sg.nblk = mb.nblk;
            sg.first_cta = tg.nclusters;
            tg.nclusters += mb.nb * mb.nblk;
            segs.push_back(sg);
            tg.members.push_back(mb.i);
            FinalSeg f{};
            f.block = sg.block;
            f.out = (double*)t_out2_.ptr + ooff;
            f.nblk = mb.nblk;
            f.nout = 2 * mb.nb;
            f.first_out = (int)ooff;
            fin.push_back(f);
            out_of.emplace_back(mb.i, ooff);
            boff += (size_t)2 * mb.nb * mb.nblk;
            ooff += (size_t)2 * mb.nb;
        }
        tg.off = append(segtab, segs);
        tg.nseg = (int)segs.size();
        tgl.push_back(tg);
    }
    const size_t foff = append(segtab, fin);
    CK(t_b_.upload(segtab.data(), segtab.size(), stream_));
    for (const G& g : gl)
        CK(LAUNCH(launch_deriv4_batch, (const DerivSeg*)((unsigned char*)t_b_.ptr + g.off),
                  g.nseg, g.ncta, g.C, stream_));
    for (const TG& g : tgl) {
        CK(launch_deriv_tc_batch((const DerivSeg*)((unsigned char*)t_b_.ptr + g.off), g.nseg,
                                 g.nclusters, g.d, stream_));
        for (int i : g.members) m_[i]->tc_used_ = true;
    }
    CK(launch_final_batch((const FinalSeg*)((unsigned char*)t_b_.ptr + foff), (int)fin.size(),
                          (int)ooff, stream_));
    double* h = stage(ooff);
    if (!h) return kErrOOM;
    CK(cudaMemcpyAsync(h, t_out2_.ptr, sizeof(double) * ooff, cudaMemcpyDeviceToHost, stream_));
    for (const auto& mo : out_of) {
        const int i = mo.first, nb = counts[i];
        if (sums[i]) push_pending(Pending{h + mo.second, sums[i], (size_t)nb, -1});
        if (sumsq[i]) push_pending(Pending{h + mo.second + nb, sumsq[i], (size_t)nb, -1});
    }
    if (deferred()) return kSuccess;   // delivered by wait()
    return sync();
}

// ------------------------------------- fused pre-order walk + derivatives
// Per member, updatePrePartialsWithDerivatives(ops, post, dmat, cw): the
// pre-order walk and the edge derivatives of its branches, sums in op order.
// 4-state members with 1, 2, 4 or 8 categories run the batched fused walk
// (one launch per category count); FP32 members with 4 < S <= 64 run the
// batched tensor-core fused walk (one launch per (S, C) group); any other
// member, or a list the fused walks cannot take, runs its own call on the
// shared stream.
int Batch::preDerivatives(const int* const* ops, const int* counts, const int* const* post,
                          const int* const* dmat, const int* cw, double* const* sums,
                          double* const* sumsq) {
    const int n = size();
    struct Member {
        int i;
        size_t a_off;     // fused op list (S = 4) or walk table (tensor cores)
        size_t d_off;     // derivative table (tensor cores)
        int nops;
    };
    std::map<int, std::vector<Member>> groups;                           // C -> 4-state
    std::map<std::tuple<int, int, int>, std::vector<Member>> tcgroups;   // (S, Sg, C)
    std::map<std::tuple<int, int, int>, bool> tcpairs;   // every member's list all sibling pairs
    std::vector<unsigned char> table;
    std::vector<int> fallback;
    for (int i = 0; i < n; ++i) {
        Instance* in = m_[i];
        if (counts[i] < 0) return kErrRange;
        if (counts[i] == 0) continue;
        std::vector<OpDesc> tab;
        std::vector<DerivDesc> dtab;
        std::vector<PreDerivOp> fops;
        bool idem = false;
        const int rc = in->build_prederiv(ops[i], counts[i], post[i], dmat[i], &cw[i], tab, dtab,
                                          fops, idem);
        if (rc == Instance::kNotFused) {
            fallback.push_back(i);
            continue;
        }
        if (rc) return rc;
        if (in->S_ == 4) {
            if (!batched4(in, in->S_, in->C_)) {
                fallback.push_back(i);
                continue;
            }
            groups[in->C_].push_back(Member{i, append(table, fops), 0, counts[i]});
        } else {
            const size_t a = append(table, tab);
            const auto key = std::make_tuple(in->S_, in->Sg_, in->C_);
            tcgroups[key].push_back(Member{i, a, append(table, dtab), counts[i]});
            bool pairs = counts[i] % 2 == 0;
            for (int k = 0; pairs && k < counts[i]; k += 2) pairs = (tab[k].kind & kPairFirst) != 0;
            auto it = tcpairs.find(key);
            tcpairs[key] = (it == tcpairs.end() ? true : it->second) && pairs;
        }
    }
    auto own_call = [&](int i) {
        return m_[i]->updatePrePartialsWithDerivatives(ops[i], counts[i], post[i], dmat[i], &cw[i],
                                                       sums[i], sumsq[i]);
    };
    for (int i : fallback) {
        const int rc = own_call(i);
        if (rc) return rc;
    }
    if (groups.empty() && tcgroups.empty()) return kSuccess;
    CK(t_a_.upload(table.data(), table.size(), stream_));
    auto nblk_of = [&](const Instance* in) {
        return in->S_ == 4 ? ceil_div(in->Pp_, pre_deriv4_batch_patterns(in->C_)) * 8
                           : in->Pp_ / tc_tile_patterns();
    };
    size_t blocks = 0, outs = 0;
    for (auto* grp : {&groups})
        for (auto& kv : *grp)
            for (const Member& mb : kv.second) {
                blocks += (size_t)2 * mb.nops * nblk_of(m_[mb.i]);
                outs += (size_t)2 * mb.nops;
            }
    for (auto& kv : tcgroups)
        for (const Member& mb : kv.second) {
            blocks += (size_t)2 * mb.nops * nblk_of(m_[mb.i]);
            outs += (size_t)2 * mb.nops;
        }
    CK(t_block_.reserve(sizeof(double) * blocks));
    CK(t_out2_.reserve(sizeof(double) * outs));
    std::vector<unsigned char> segtab;
    std::vector<FinalSeg> fin;
    std::vector<std::pair<int, size_t>> out_of;   // (member, first output) in t_out2_
    size_t boff = 0, ooff = 0;
    auto seg_of = [&](const Member& mb, int first) {
        Instance* in = m_[mb.i];
        PreDerivSeg sg{};
        const unsigned char* base = (const unsigned char*)t_a_.ptr;
        if (in->S_ == 4) {
            sg.fops = (const PreDerivOp*)(base + mb.a_off);
        } else {
            sg.ops = (const OpDesc*)(base + mb.a_off);
            sg.dds = (const DerivDesc*)(base + mb.d_off);
        }
        sg.catw = in->d_catw_ + (size_t)cw[mb.i] * in->C_;
        sg.patw = in->d_patw_;
        sg.block = (double*)t_block_.ptr + boff;
        sg.nops = mb.nops;
        sg.P = in->P_;
        sg.Pp = in->Pp_;
        sg.nblk = nblk_of(in);
        sg.log_scalers = (int)in->log_scalers_;
        sg.first_cta = first;
        FinalSeg f{};
        f.block = sg.block;
        f.out = (double*)t_out2_.ptr + ooff;
        f.nblk = sg.nblk;
        f.nout = 2 * mb.nops;
        f.first_out = (int)ooff;
        fin.push_back(f);
        out_of.emplace_back(mb.i, ooff);
        boff += (size_t)2 * mb.nops * sg.nblk;
        ooff += (size_t)2 * mb.nops;
        return sg;
    };
    struct G {
        int C;
        size_t off;
        int nseg;
        int ncta;
    };
    std::vector<G> gl;
    for (auto& kv : groups) {
        std::vector<PreDerivSeg> segs;
        int cta = 0;
        for (const Member& mb : kv.second) {
            segs.push_back(seg_of(mb, cta));
            cta += ceil_div(m_[mb.i]->Pp_, pre_deriv4_batch_patterns(kv.first));
        }
        gl.push_back(G{kv.first, append(segtab, segs), (int)segs.size(), cta});
    }
    struct TG {
        Dims d;
        size_t off;
        int nseg;
        int ntiles;
        bool pairs;
        std::vector<int> members;
    };
    std::vector<TG> tgl;
    for (auto& kv : tcgroups) {
        std::vector<PreDerivSeg> segs;
        TG tg{};
        tg.d = Dims{std::get<0>(kv.first), std::get<1>(kv.first), 0, 0, std::get<2>(kv.first)};
        tg.pairs = tcpairs[kv.first];
        for (const Member& mb : kv.second) {
            segs.push_back(seg_of(mb, tg.ntiles));
            tg.ntiles += m_[mb.i]->Pp_ / tc_tile_patterns();
            tg.members.push_back(mb.i);
        }
        tg.off = append(segtab, segs);
        tg.nseg = (int)segs.size();
        tgl.push_back(tg);
    }
    const size_t foff = append(segtab, fin);
    CK(t_b_.upload(segtab.data(), segtab.size(), stream_));
    // the tensor-core groups on the second stream, beside the 4-state ones
    const bool split = !gl.empty() && !tgl.empty();
    if (split) CK(fork());
    cudaStream_t ts = split ? side_ : stream_;
    cudaError_t err = cudaSuccess;
    std::vector<int> late;   // tensor-core groups that cannot launch here: own calls
    for (const TG& g : tgl) {
        // the sibling-pair form where every member's list is made of pairs
        // and the width has it (17 to 32 padded states), else the op walk
        const PreDerivSeg* segs = (const PreDerivSeg*)((unsigned char*)t_b_.ptr + g.off);
        cudaError_t e = cudaErrorInvalidValue;
        if (g.pairs) e = launch_prederiv_tc_pairs_batch(segs, g.nseg, g.ntiles, g.d, ts);
        if (e == cudaErrorInvalidValue) {
            (void)cudaGetLastError();
            e = launch_prederiv_tc_batch(segs, g.nseg, g.ntiles, g.d, ts);
        }
        if (e == cudaErrorInvalidConfiguration) {
            (void)cudaGetLastError();
            late.insert(late.end(), g.members.begin(), g.members.end());
            continue;
        }
        if (e != cudaSuccess) err = e;
        for (int i : g.members) m_[i]->tc_used_ = true;
    }
    for (const G& g : gl) {
        if (err != cudaSuccess) break;
        err = LAUNCH(launch_pre_deriv4_batch,
                     (const PreDerivSeg*)((unsigned char*)t_b_.ptr + g.off), g.nseg, g.ncta, g.C,
                     stream_);
    }
    if (split) {
        const cudaError_t e = join();
        if (err == cudaSuccess) err = e;
    }
    CK(err);
    CK(launch_final_batch((const FinalSeg*)((unsigned char*)t_b_.ptr + foff), (int)fin.size(),
                          (int)ooff, stream_));
    double* h = stage(ooff);
    if (!h) return kErrOOM;
    CK(cudaMemcpyAsync(h, t_out2_.ptr, sizeof(double) * ooff, cudaMemcpyDeviceToHost, stream_));
    for (const auto& mo : out_of) {
        const int i = mo.first, nb = counts[i];
        if (std::find(late.begin(), late.end(), i) != late.end()) continue;
        if (sums[i]) push_pending(Pending{h + mo.second, sums[i], (size_t)nb, -1});
        if (sumsq[i]) push_pending(Pending{h + mo.second + nb, sumsq[i], (size_t)nb, -1});
    }
    for (int i : late) {
        const int rc = own_call(i);
        if (rc) return rc;
    }
    if (deferred()) return kSuccess;   // delivered by wait()
    return sync();
}

}  // namespace b200
