// extern "C" entry points of libbeagle_b200.so (declared in
// include/beagle_b200.h).  Each forwards to the instance's method, the way the
// reference dispatcher forwards beagle.h calls to a BeagleImpl
// (libhmsbeagle/beagle.cpp:744-1865), but with a bounds-checked instance table
// and no exception ever crossing the C boundary.
#include "beagle_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "b200_batch.h"
#include "b200_instance.h"

namespace {

std::mutex g_mu;
std::vector<std::unique_ptr<b200::Instance>> g_instances;
std::vector<std::unique_ptr<b200::Batch>> g_batches;
std::vector<std::vector<int>> g_batch_members;   // instance handles of each batch
std::vector<BeagleB200Resource> g_resources;
std::vector<std::string> g_resource_names;
BeagleB200ResourceList g_resource_list{nullptr, 0};

b200::Instance* get(int h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h < 0 || h >= (int)g_instances.size()) return nullptr;
    return g_instances[h].get();
}

// Run one instance method with the instance's device current; exceptions and
// a missing instance become return codes.
template <typename F>
int call(int h, F&& f) {
    b200::Instance* in = get(h);
    if (!in) return BEAGLE_B200_ERROR_UNINITIALIZED_INSTANCE;
    try {
        if (cudaSetDevice(in->device()) != cudaSuccess) return BEAGLE_B200_ERROR_GENERAL;
        return f(in);
    } catch (const std::bad_alloc&) {
        return BEAGLE_B200_ERROR_OUT_OF_MEMORY;
    } catch (...) {
        return BEAGLE_B200_ERROR_UNIDENTIFIED_EXCEPTION;
    }
}

// Run one batch method with the batch's device current, after checking that
// every member instance still exists.
template <typename F>
int call_batch(int h, F&& f) {
    b200::Batch* bt = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (h < 0 || h >= (int)g_batches.size() || !g_batches[h])
            return BEAGLE_B200_ERROR_UNINITIALIZED_INSTANCE;
        for (int m : g_batch_members[h])
            if (m < 0 || m >= (int)g_instances.size() || !g_instances[m])
                return BEAGLE_B200_ERROR_UNINITIALIZED_INSTANCE;
        bt = g_batches[h].get();
    }
    try {
        b200::Instance* first = get(g_batch_members[h][0]);
        if (!first || cudaSetDevice(first->device()) != cudaSuccess)
            return BEAGLE_B200_ERROR_GENERAL;
        return f(bt);
    } catch (const std::bad_alloc&) {
        return BEAGLE_B200_ERROR_OUT_OF_MEMORY;
    } catch (...) {
        return BEAGLE_B200_ERROR_UNIDENTIFIED_EXCEPTION;
    }
}

constexpr long kSupportFlags =
    BEAGLE_B200_FLAG_PRECISION_SINGLE | BEAGLE_B200_FLAG_PRECISION_DOUBLE |
    BEAGLE_B200_FLAG_COMPUTATION_SYNCH | BEAGLE_B200_FLAG_COMPUTATION_ASYNCH |
    BEAGLE_B200_FLAG_EIGEN_REAL | BEAGLE_B200_FLAG_SCALING_MANUAL |
    BEAGLE_B200_FLAG_SCALERS_RAW | BEAGLE_B200_FLAG_SCALERS_LOG | BEAGLE_B200_FLAG_VECTOR_NONE |
    BEAGLE_B200_FLAG_THREADING_NONE | BEAGLE_B200_FLAG_PROCESSOR_GPU |
    BEAGLE_B200_FLAG_INVEVEC_STANDARD | BEAGLE_B200_FLAG_INVEVEC_TRANSPOSED |
    BEAGLE_B200_FLAG_FRAMEWORK_CUDA | BEAGLE_B200_FLAG_PARALLELOPS_GRID |
    BEAGLE_B200_FLAG_PREORDER_TRANSPOSE_MANUAL | BEAGLE_B200_FLAG_PREORDER_TRANSPOSE_AUTO;

}  // namespace

extern "C" {

const char* beagleB200GetVersion(void) { return "beagle-b200 1.0 (BEAGLE 4.0.1 API)"; }

BeagleB200ResourceList* beagleB200GetResourceList(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    static bool listed = false;
    if (!listed) {
        listed = true;
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            (void)cudaGetLastError();
            n = 0;
        }
        // One entry per CUDA device, entry k = device ordinal k.  Devices the
        // sm_100a kernels cannot run on are listed with no support flags.
        std::vector<long> support;
        for (int d = 0; d < n; ++d) {
            cudaDeviceProp prop;
            if (cudaGetDeviceProperties(&prop, d) != cudaSuccess) {
                (void)cudaGetLastError();
                prop.major = prop.minor = 0;
                prop.name[0] = 0;
            }
            g_resource_names.push_back(std::string(prop.name) + " (sm_" +
                                       std::to_string(prop.major) + std::to_string(prop.minor) +
                                       "), device " + std::to_string(d));
            support.push_back(prop.major == 10 && prop.minor == 0 ? kSupportFlags : 0L);
        }
        g_resources.resize(g_resource_names.size());
        for (size_t k = 0; k < g_resources.size(); ++k) {
            g_resources[k].name = const_cast<char*>(g_resource_names[k].c_str());
            g_resources[k].description = const_cast<char*>("B200 likelihood kernels (sm_100a)");
            g_resources[k].supportFlags = support[k];
            g_resources[k].requiredFlags = BEAGLE_B200_FLAG_FRAMEWORK_CUDA;
        }
        g_resource_list.list = g_resources.empty() ? nullptr : g_resources.data();
        g_resource_list.length = (int)g_resources.size();
    }
    return &g_resource_list;
}

int beagleB200CreateInstance(int tipCount, int partialsBufferCount, int compactBufferCount,
                             int stateCount, int patternCount, int eigenBufferCount,
                             int matrixBufferCount, int categoryCount, int scaleBufferCount,
                             int* resourceList, int resourceCount, long preferenceFlags,
                             long requirementFlags, BeagleB200InstanceDetails* returnInfo) {
    try {
        const int device = (resourceList && resourceCount > 0) ? resourceList[0] : 0;
        std::unique_ptr<b200::Instance> in(new b200::Instance());
        const int rc = in->create(tipCount, partialsBufferCount, compactBufferCount, stateCount,
                                  patternCount, eigenBufferCount, matrixBufferCount,
                                  categoryCount, scaleBufferCount, device, preferenceFlags,
                                  requirementFlags);
        if (rc != 0) return rc;
        if (returnInfo) {
            returnInfo->resourceNumber = device;
            returnInfo->resourceName = const_cast<char*>("B200 (sm_100a)");
            returnInfo->implName = const_cast<char*>(in->implName());
            returnInfo->implDescription =
                const_cast<char*>("op-walking sm_100a kernels, FP64 P(t) and reductions");
            returnInfo->flags = in->flags();
        }
        std::lock_guard<std::mutex> lk(g_mu);
        for (size_t k = 0; k < g_instances.size(); ++k)
            if (!g_instances[k]) {
                g_instances[k] = std::move(in);
                return (int)k;
            }
        g_instances.push_back(std::move(in));
        return (int)g_instances.size() - 1;
    } catch (const std::bad_alloc&) {
        return BEAGLE_B200_ERROR_OUT_OF_MEMORY;
    } catch (...) {
        return BEAGLE_B200_ERROR_UNIDENTIFIED_EXCEPTION;
    }
}

int beagleB200FinalizeInstance(int instance) {
    std::unique_ptr<b200::Instance> victim;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (instance < 0 || instance >= (int)g_instances.size() || !g_instances[instance])
            return BEAGLE_B200_ERROR_UNINITIALIZED_INSTANCE;
        victim = std::move(g_instances[instance]);
    }
    victim.reset();
    return BEAGLE_B200_SUCCESS;
}

int beagleB200Finalize(void) {
    std::vector<std::unique_ptr<b200::Instance>> all;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        all.swap(g_instances);
    }
    all.clear();
    return BEAGLE_B200_SUCCESS;
}

int beagleB200SetCPUThreadCount(int instance, int) {
    return call(instance, [](b200::Instance*) { return BEAGLE_B200_ERROR_NO_IMPLEMENTATION; });
}

int beagleB200SetTipStates(int h, int tip, const int* s) {
    return call(h, [&](b200::Instance* in) { return in->setTipStates(tip, s); });
}
int beagleB200SetTipPartials(int h, int tip, const double* p) {
    return call(h, [&](b200::Instance* in) { return in->setTipPartials(tip, p); });
}
int beagleB200SetRootPrePartials(int h, const int* b, const int* f, int n) {
    return call(h, [&](b200::Instance* in) { return in->setRootPrePartials(b, f, n); });
}
int beagleB200SetPartials(int h, int b, const double* p) {
    return call(h, [&](b200::Instance* in) { return in->setPartials(b, p); });
}
int beagleB200GetPartials(int h, int b, int s, double* o) {
    return call(h, [&](b200::Instance* in) { return in->getPartials(b, s, o); });
}
int beagleB200SetEigenDecomposition(int h, int e, const double* v, const double* iv,
                                    const double* ev) {
    return call(h, [&](b200::Instance* in) { return in->setEigenDecomposition(e, v, iv, ev); });
}
int beagleB200SetStateFrequencies(int h, int i, const double* f) {
    return call(h, [&](b200::Instance* in) { return in->setStateFrequencies(i, f); });
}
int beagleB200SetCategoryWeights(int h, int i, const double* w) {
    return call(h, [&](b200::Instance* in) { return in->setCategoryWeights(i, w); });
}
int beagleB200SetCategoryRates(int h, const double* r) {
    return call(h, [&](b200::Instance* in) { return in->setCategoryRates(r); });
}
int beagleB200SetCategoryRatesWithIndex(int h, int i, const double* r) {
    return call(h, [&](b200::Instance* in) { return in->setCategoryRatesWithIndex(i, r); });
}
int beagleB200SetPatternWeights(int h, const double* w) {
    return call(h, [&](b200::Instance* in) { return in->setPatternWeights(w); });
}
int beagleB200SetPatternPartitions(int h, int n, const int* p) {
    return call(h, [&](b200::Instance* in) { return in->setPatternPartitions(n, p); });
}

int beagleB200ConvolveTransitionMatrices(int h, const int* a, const int* b, const int* r, int n) {
    return call(h, [&](b200::Instance* in) { return in->convolveTransitionMatrices(a, b, r, n); });
}
int beagleB200AddTransitionMatrices(int h, const int*, const int*, const int*, int) {
    return call(h, [](b200::Instance*) { return BEAGLE_B200_ERROR_NO_IMPLEMENTATION; });
}
int beagleB200TransposeTransitionMatrices(int h, const int* a, const int* r, int n) {
    return call(h, [&](b200::Instance* in) { return in->transposeTransitionMatrices(a, r, n); });
}
int beagleB200UpdateTransitionMatrices(int h, int e, const int* p, const int* d1, const int* d2,
                                       const double* t, int n) {
    return call(h, [&](b200::Instance* in) {
        return in->updateTransitionMatrices(e, p, d1, d2, t, n);
    });
}
int beagleB200UpdateTransitionMatricesWithModelCategories(int h, int* e, const int* p,
                                                          const int* d1, const int* d2,
                                                          const double* t, int n) {
    return call(h, [&](b200::Instance* in) {
        return in->updateTransitionMatricesWithModelCategories(e, p, d1, d2, t, n);
    });
}
int beagleB200UpdateTransitionMatricesWithMultipleModels(int h, const int* e, const int* r,
                                                         const int* p, const int* d1,
                                                         const int* d2, const double* t, int n) {
    return call(h, [&](b200::Instance* in) {
        return in->updateTransitionMatricesWithMultipleModels(e, r, p, d1, d2, t, n);
    });
}
int beagleB200SetTransitionMatrix(int h, int m, const double* v, double pad) {
    return call(h, [&](b200::Instance* in) { return in->setTransitionMatrix(m, v, pad); });
}
int beagleB200SetDifferentialMatrix(int h, int m, const double* v) {
    return call(h, [&](b200::Instance* in) { return in->setTransitionMatrix(m, v, 0.0); });
}
int beagleB200GetTransitionMatrix(int h, int m, double* o) {
    return call(h, [&](b200::Instance* in) { return in->getTransitionMatrix(m, o); });
}
int beagleB200SetTransitionMatrices(int h, const int* m, const double* v, const double* pads,
                                    int n) {
    return call(h, [&](b200::Instance* in) { return in->setTransitionMatrices(m, v, pads, n); });
}

int beagleB200UpdatePartials(const int h, const BeagleB200Operation* ops, int n, int cum) {
    return call(h, [&](b200::Instance* in) {
        return in->updatePartials(reinterpret_cast<const int*>(ops), n, cum);
    });
}
int beagleB200UpdatePrePartials(const int h, const BeagleB200Operation* ops, int n, int cum) {
    return call(h, [&](b200::Instance* in) {
        return in->updatePrePartials(reinterpret_cast<const int*>(ops), n, cum);
    });
}
int beagleB200UpdatePartialsByPartition(const int h, const BeagleB200OperationByPartition* ops,
                                        int n) {
    return call(h, [&](b200::Instance* in) {
        return in->updatePartialsByPartition(reinterpret_cast<const int*>(ops), n);
    });
}
int beagleB200UpdatePrePartialsByPartition(const int h,
                                           const BeagleB200OperationByPartition* ops, int n) {
    return call(h, [&](b200::Instance* in) {
        return in->updatePrePartialsByPartition(reinterpret_cast<const int*>(ops), n);
    });
}
int beagleB200WaitForPartials(const int h, const int*, int) {
    return call(h, [&](b200::Instance* in) { return in->waitForPartials(); });
}

int beagleB200AccumulateScaleFactors(int h, const int* idx, int n, int cum) {
    return call(h, [&](b200::Instance* in) {
        return in->accumulateScaleFactors(idx, n, cum, 1.0, -1);
    });
}
int beagleB200AccumulateScaleFactorsByPartition(int h, const int* idx, int n, int cum, int part) {
    return call(h, [&](b200::Instance* in) {
        return part < 0 ? BEAGLE_B200_ERROR_OUT_OF_RANGE
                        : in->accumulateScaleFactors(idx, n, cum, 1.0, part);
    });
}
int beagleB200RemoveScaleFactors(int h, const int* idx, int n, int cum) {
    return call(h, [&](b200::Instance* in) {
        return in->accumulateScaleFactors(idx, n, cum, -1.0, -1);
    });
}
int beagleB200RemoveScaleFactorsByPartition(int h, const int* idx, int n, int cum, int part) {
    return call(h, [&](b200::Instance* in) {
        return part < 0 ? BEAGLE_B200_ERROR_OUT_OF_RANGE
                        : in->accumulateScaleFactors(idx, n, cum, -1.0, part);
    });
}
int beagleB200ResetScaleFactors(int h, int cum) {
    return call(h, [&](b200::Instance* in) { return in->resetScaleFactors(cum, -1); });
}
int beagleB200ResetScaleFactorsByPartition(int h, int cum, int part) {
    return call(h, [&](b200::Instance* in) {
        return part < 0 ? BEAGLE_B200_ERROR_OUT_OF_RANGE : in->resetScaleFactors(cum, part);
    });
}
int beagleB200CopyScaleFactors(int h, int dst, int src) {
    return call(h, [&](b200::Instance* in) { return in->copyScaleFactors(dst, src); });
}
int beagleB200GetScaleFactors(int h, int src, double* out) {
    return call(h, [&](b200::Instance* in) { return in->getScaleFactors(src, out); });
}

int beagleB200CalculateRootLogLikelihoods(int h, const int* b, const int* w, const int* f,
                                          const int* c, int n, double* out) {
    return call(h, [&](b200::Instance* in) {
        return in->calculateRootLogLikelihoods(b, w, f, c, n, out);
    });
}
int beagleB200CalculateRootLogLikelihoodsByPartition(int h, const int* b, const int* w,
                                                     const int* f, const int* c, const int* p,
                                                     int np, int n, double* byp, double* out) {
    return call(h, [&](b200::Instance* in) {
        return in->calculateRootLogLikelihoodsByPartition(b, w, f, c, p, np, n, byp, out);
    });
}
int beagleB200CalculateEdgeDerivatives(int h, const int* post, const int* pre, const int* d,
                                       const int* w, int n, double* o, double* s, double* sq) {
    return call(h, [&](b200::Instance* in) {
        return in->calculateEdgeDerivatives(post, pre, d, w, n, o, s, sq);
    });
}
int beagleB200UpdatePartialsWithRootLogLikelihood(int h, const int* ops, int count,
                                                   int cumulative, int root, int cw, int sf,
                                                   double* out) {
    return call(h, [&](b200::Instance* in) {
        return in->updatePartialsWithRootLogLikelihood(ops, count, cumulative, root, cw, sf, out);
    });
}
int beagleB200UpdatePrePartialsWithDerivatives(int h, const int* ops, int count,
                                               const int* post, const int* dmat, const int* cw,
                                               double* s, double* sq) {
    return call(h, [&](b200::Instance* in) {
        return in->updatePrePartialsWithDerivatives(ops, count, post, dmat, cw, s, sq);
    });
}
int beagleB200GetTunedVariants(int h, int* out) {
    if (!out) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call(h, [&](b200::Instance* in) {
        for (int k = 0; k < 4; ++k) out[k] = in->picked(k + 1);
        return BEAGLE_B200_SUCCESS;
    });
}
int beagleB200CalculateCrossProductDerivative(int h, const int* post, const int* pre,
                                              const int* rates, const int* w, const double* t,
                                              int n, double* sum, double* sumsq) {
    (void)sumsq;   // not written, as in the reference CPU implementation
    return call(h, [&](b200::Instance* in) {
        return in->calculateCrossProducts(post, pre, rates, w, t, n, sum);
    });
}
int beagleB200CalculateEdgeLogLikelihoods(int h, const int* pa, const int* ch, const int* pm,
                                          const int* d1, const int* d2, const int* w,
                                          const int* f, const int* c, int n, double* o,
                                          double* o1, double* o2) {
    return call(h, [&](b200::Instance* in) {
        return in->calculateEdgeLogLikelihoods(pa, ch, pm, d1, d2, w, f, c, n, o, o1, o2);
    });
}
int beagleB200CalculateEdgeLogLikelihoodsByPartition(
    int h, const int* pa, const int* ch, const int* pm, const int* d1, const int* d2,
    const int* w, const int* f, const int* c, const int* parts, int np, int n, double* byp,
    double* o, double* d1byp, double* o1, double* d2byp, double* o2) {
    return call(h, [&](b200::Instance* in) {
        return in->calculateEdgeLogLikelihoodsByPartition(pa, ch, pm, d1, d2, w, f, c, parts, np,
                                                          n, byp, o, d1byp, o1, d2byp, o2);
    });
}
int beagleB200GetLogLikelihood(int h, double* o) {
    return call(h, [&](b200::Instance* in) { return in->getLogLikelihood(o); });
}
int beagleB200GetDerivatives(int h, double* d1, double* d2) {
    return call(h, [&](b200::Instance* in) { return in->getDerivatives(d1, d2); });
}
int beagleB200GetSiteLogLikelihoods(int h, double* o) {
    return call(h, [&](b200::Instance* in) { return in->getSiteLogLikelihoods(o); });
}
int beagleB200GetSiteDerivatives(int h, double* d1, double* d2) {
    return call(h, [&](b200::Instance* in) { return in->getSiteDerivatives(d1, d2); });
}

int beagleB200GetCudaStream(int h, void** out) {
    return call(h, [&](b200::Instance* in) {
        if (!out) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
        *out = (void*)in->stream();
        return BEAGLE_B200_SUCCESS;
    });
}


int beagleB200InjectKernelTimeout(int h, int which) {
    return call(h, [&](b200::Instance* in) { return in->injectKernelTimeout(which); });
}

int beagleB200CreateBatch(const int* instances, int count) {
    if (!instances || count <= 0) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    std::vector<b200::Instance*> members;
    std::vector<int> handles(instances, instances + count);
    for (int h : handles) {
        b200::Instance* in = get(h);
        if (!in) return BEAGLE_B200_ERROR_UNINITIALIZED_INSTANCE;
        members.push_back(in);
    }
    {
        // an instance belongs to at most one batch
        std::lock_guard<std::mutex> lk(g_mu);
        for (size_t b = 0; b < g_batch_members.size(); ++b)
            if (g_batches[b])
                for (int h : g_batch_members[b])
                    if (std::find(handles.begin(), handles.end(), h) != handles.end())
                        return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    }
    try {
        if (cudaSetDevice(members[0]->device()) != cudaSuccess) return BEAGLE_B200_ERROR_GENERAL;
        std::unique_ptr<b200::Batch> bt(new b200::Batch());
        const int rc = bt->create(members);
        if (rc) return rc;
        std::lock_guard<std::mutex> lk(g_mu);
        for (size_t k = 0; k < g_batches.size(); ++k)
            if (!g_batches[k]) {
                g_batches[k] = std::move(bt);
                g_batch_members[k] = handles;
                return (int)k;
            }
        g_batches.push_back(std::move(bt));
        g_batch_members.push_back(handles);
        return (int)g_batches.size() - 1;
    } catch (const std::bad_alloc&) {
        return BEAGLE_B200_ERROR_OUT_OF_MEMORY;
    } catch (...) {
        return BEAGLE_B200_ERROR_UNIDENTIFIED_EXCEPTION;
    }
}

int beagleB200FinalizeBatch(int batch) {
    std::unique_ptr<b200::Batch> bt;
    std::vector<int> members;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (batch < 0 || batch >= (int)g_batches.size() || !g_batches[batch])
            return BEAGLE_B200_ERROR_UNINITIALIZED_INSTANCE;
        bt = std::move(g_batches[batch]);
        members = g_batch_members[batch];
        g_batch_members[batch].clear();
    }
    // Members that were finalized meanwhile are skipped: release only the live ones.
    b200::Instance* first = members.empty() ? nullptr : get(members[0]);
    if (first) cudaSetDevice(first->device());
    bool all_alive = true;
    for (int h : members) all_alive = all_alive && get(h) != nullptr;
    if (all_alive) bt->release();
    bt.reset();
    return BEAGLE_B200_SUCCESS;
}

int beagleB200BatchUpdateTransitionMatrices(int batch, const int* eig, const int* const* prob,
                                            const double* const* t, const int* counts) {
    if (!prob || !t || !counts) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) {
        return b->updateTransitionMatrices(eig, prob, t, counts);
    });
}

int beagleB200BatchUpdatePartials(int batch, const int* const* ops, const int* counts,
                                  const int* cumulative) {
    if (!ops || !counts) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) {
        return b->updatePartials(ops, counts, cumulative, false);
    });
}

int beagleB200BatchUpdatePrePartials(int batch, const int* const* ops, const int* counts) {
    if (!ops || !counts) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) {
        return b->updatePartials(ops, counts, nullptr, true);
    });
}

int beagleB200BatchAccumulateScaleFactors(int batch, const int* const* idx, const int* counts,
                                          const int* cumulative, int reset) {
    if (!idx || !counts || !cumulative) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) {
        return b->accumulateScaleFactors(idx, counts, cumulative, reset);
    });
}

int beagleB200BatchSetRootPrePartials(int batch, const int* bufs, const int* freqs) {
    if (!bufs || !freqs) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) { return b->setRootPrePartials(bufs, freqs); });
}

int beagleB200BatchCalculateRootLogLikelihoods(int batch, const int* bufs, const int* cw,
                                               const int* sf, const int* cum, double* out) {
    if (!bufs || !cw || !sf || !out) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) {
        return b->rootLogLikelihoods(bufs, cw, sf, cum, out);
    });
}

int beagleB200BatchUpdatePartialsWithRootLogLikelihood(int batch, const int* const* ops,
                                                        const int* counts, const int* cumulative,
                                                        const int* roots, const int* cw,
                                                        const int* sf, double* out) {
    if (!ops || !counts || !cumulative || !roots || !cw || !sf || !out)
        return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) {
        return b->postRoot(ops, counts, cumulative, roots, cw, sf, out);
    });
}

int beagleB200BatchCalculateEdgeDerivatives(int batch, const int* const* post,
                                            const int* const* pre, const int* const* dmat,
                                            const int* cw, const int* counts,
                                            double* const* sums, double* const* sumsq) {
    if (!post || !pre || !dmat || !cw || !counts || !sums || !sumsq)
        return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) {
        return b->edgeDerivatives(post, pre, dmat, cw, counts, sums, sumsq);
    });
}

int beagleB200BatchUpdatePrePartialsWithDerivatives(int batch, const int* const* operations,
                                                    const int* counts,
                                                    const int* const* postBufferIndices,
                                                    const int* const* derivativeMatrixIndices,
                                                    const int* categoryWeightsIndices,
                                                    double* const* outSumDerivatives,
                                                    double* const* outSumSquaredDerivatives) {
    if (!operations || !counts || !postBufferIndices || !derivativeMatrixIndices ||
        !categoryWeightsIndices || !outSumDerivatives || !outSumSquaredDerivatives)
        return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) {
        return b->preDerivatives(operations, counts, postBufferIndices, derivativeMatrixIndices,
                                 categoryWeightsIndices, outSumDerivatives,
                                 outSumSquaredDerivatives);
    });
}

int beagleB200BatchLaunchGraphWithLengths(int batch, int graph, const double* lengths,
                                          int count) {
    return call_batch(batch, [&](b200::Batch* b) {
        return b->launchGraphWithLengths(graph, lengths, count);
    });
}

int beagleB200BatchBeginCapture(int batch) {
    return call_batch(batch, [&](b200::Batch* b) { return b->beginCapture(); });
}

int beagleB200BatchEndCapture(int batch, int* graph) {
    if (!graph) return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    return call_batch(batch, [&](b200::Batch* b) { return b->endCapture(graph); });
}

int beagleB200BatchLaunchGraph(int batch, int graph) {
    return call_batch(batch, [&](b200::Batch* b) { return b->launchGraph(graph); });
}

int beagleB200BatchWait(int batch) {
    return call_batch(batch, [&](b200::Batch* b) { return b->wait(); });
}

int beagleB200BeginCapture(int instance) {
    return call(instance, [&](b200::Instance* in) { return in->beginCapture(); });
}

int beagleB200EndCapture(int instance, int* graph) {
    return call(instance, [&](b200::Instance* in) { return in->endCapture(graph); });
}

int beagleB200LaunchGraph(int instance, int graph) {
    return call(instance, [&](b200::Instance* in) { return in->launchGraph(graph); });
}

int beagleB200LaunchGraphWithLengths(int instance, int graph, const double* lengths, int count) {
    return call(instance, [&](b200::Instance* in) {
        return in->launchGraphWithLengths(graph, lengths, count);
    });
}

}  // extern "C"
