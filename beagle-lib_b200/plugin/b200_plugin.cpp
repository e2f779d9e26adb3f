// libhmsbeagle-cuda.so.40.0.0: the B200 resource as a plugin of the stock
// BEAGLE dispatcher (libhmsbeagle.so).
//
// The dispatcher dlopens "libhmsbeagle-cuda.so.40.0.0" by name
// (libhmsbeagle/beagle.cpp:161, libhmsbeagle/plugin/UnixSharedLibrary.h:40-58),
// calls its extern "C" plugin_init (libhmsbeagle/plugin/Plugin.cpp:31-34),
// lists getBeagleResources() / getBeagleFactories()
// (libhmsbeagle/plugin/Plugin.h:63-64), ranks resource x factory pairs by
// flags (libhmsbeagle/beagle.cpp:341-460) and calls
// BeagleImplFactory::createImpl (libhmsbeagle/BeagleImpl.h:270-290).  Every
// later beagle* call lands on a BeagleImpl virtual (BeagleImpl.h:31-268).
//
// Those are C++ interfaces (vtable order, std::list / std::string members), so
// this file is compiled against the dispatcher's own public headers with the
// same compiler; nothing of the dispatcher is reimplemented here.  Each
// virtual forwards to the C ABI of libbeagle_b200.so (include/beagle_b200.h),
// whose flag values, operation layouts and return codes are beagle.h's.
#include "libhmsbeagle/BeagleImpl.h"
#include "libhmsbeagle/beagle.h"
#include "libhmsbeagle/plugin/Plugin.h"

#include "beagle_b200.h"

#include <new>
#include <vector>

namespace b200plugin {

// BeagleB200InstanceDetails / BeagleB200Operation mirror beagle.h's structs
// member for member; the casts below rely on that.
static_assert(sizeof(BeagleB200Operation) == sizeof(BeagleOperation), "operation layout");
static_assert(sizeof(BeagleB200OperationByPartition) == sizeof(BeagleOperationByPartition),
              "partition operation layout");
static_assert(BEAGLE_B200_FLAG_FRAMEWORK_CUDA == BEAGLE_FLAG_FRAMEWORK_CUDA, "flag values");
static_assert(BEAGLE_B200_FLAG_PRECISION_SINGLE == BEAGLE_FLAG_PRECISION_SINGLE, "flag values");
static_assert(BEAGLE_B200_FLAG_PRECISION_DOUBLE == BEAGLE_FLAG_PRECISION_DOUBLE, "flag values");

class B200Impl final : public beagle::BeagleImpl {
public:
    explicit B200Impl(long precision) : precision_(precision) {}
    ~B200Impl() override {
        if (h_ >= 0) beagleB200FinalizeInstance(h_);
    }

    int createInstance(int tipCount, int partialsBufferCount, int compactBufferCount,
                       int stateCount, int patternCount, int eigenBufferCount,
                       int matrixBufferCount, int categoryCount, int scaleBufferCount,
                       int resource, int pluginResource, long preferenceFlags,
                       long requirementFlags) override {
        // This factory's precision wins over the caller's preference; a
        // requirement of the other precision never reaches it (the
        // dispatcher filters factories by requirement flags).
        const long prec = BEAGLE_FLAG_PRECISION_SINGLE | BEAGLE_FLAG_PRECISION_DOUBLE;
        preferenceFlags = (preferenceFlags & ~prec) | precision_;
        requirementFlags &= ~(prec & ~precision_);
        int device = pluginResource;
        BeagleB200InstanceDetails info;
        h_ = beagleB200CreateInstance(tipCount, partialsBufferCount, compactBufferCount,
                                      stateCount, patternCount, eigenBufferCount,
                                      matrixBufferCount, categoryCount, scaleBufferCount, &device,
                                      1, preferenceFlags, requirementFlags, &info);
        if (h_ < 0) return h_;
        resourceNumber = resource;
        flags_ = info.flags;
        impl_name_ = info.implName;
        return BEAGLE_SUCCESS;
    }

    int getInstanceDetails(BeagleInstanceDetails* out) override {
        if (out) {
            out->resourceNumber = resourceNumber;
            out->flags = flags_;
            out->implName = impl_name_;
        }
        return BEAGLE_SUCCESS;
    }

    int setCPUThreadCount(int n) override { return beagleB200SetCPUThreadCount(h_, n); }
    int setTipStates(int tip, const int* s) override { return beagleB200SetTipStates(h_, tip, s); }
    int setTipPartials(int tip, const double* p) override {
        return beagleB200SetTipPartials(h_, tip, p);
    }
    int setPartials(int b, const double* p) override { return beagleB200SetPartials(h_, b, p); }
    int setRootPrePartials(const int* b, const int* f, int n) override {
        return beagleB200SetRootPrePartials(h_, b, f, n);
    }
    int getPartials(int b, int s, double* out) override {
        return beagleB200GetPartials(h_, b, s, out);
    }
    int setEigenDecomposition(int e, const double* v, const double* iv,
                              const double* l) override {
        return beagleB200SetEigenDecomposition(h_, e, v, iv, l);
    }
    int setStateFrequencies(int i, const double* f) override {
        return beagleB200SetStateFrequencies(h_, i, f);
    }
    int setCategoryWeights(int i, const double* w) override {
        return beagleB200SetCategoryWeights(h_, i, w);
    }
    int setPatternWeights(const double* w) override { return beagleB200SetPatternWeights(h_, w); }
    int setPatternPartitions(int n, const int* p) override {
        return beagleB200SetPatternPartitions(h_, n, p);
    }
    int setCategoryRates(const double* r) override { return beagleB200SetCategoryRates(h_, r); }
    int setCategoryRatesWithIndex(int i, const double* r) override {
        return beagleB200SetCategoryRatesWithIndex(h_, i, r);
    }
    int setTransitionMatrix(int m, const double* in, double pad) override {
        return beagleB200SetTransitionMatrix(h_, m, in, pad);
    }
    int setDifferentialMatrix(int m, const double* in) override {
        return beagleB200SetDifferentialMatrix(h_, m, in);
    }
    int setTransitionMatrices(const int* m, const double* in, const double* pad,
                              int n) override {
        return beagleB200SetTransitionMatrices(h_, m, in, pad, n);
    }
    int getTransitionMatrix(int m, double* out) override {
        return beagleB200GetTransitionMatrix(h_, m, out);
    }
    int convolveTransitionMatrices(const int* a, const int* b, const int* r, int n) override {
        return beagleB200ConvolveTransitionMatrices(h_, a, b, r, n);
    }
    int addTransitionMatrices(const int* a, const int* b, const int* r, int n) override {
        return beagleB200AddTransitionMatrices(h_, a, b, r, n);
    }
    int transposeTransitionMatrices(const int* in, const int* out, int n) override {
        return beagleB200TransposeTransitionMatrices(h_, in, out, n);
    }
    int updateTransitionMatrices(int e, const int* p, const int* d1, const int* d2,
                                 const double* t, int n) override {
        return beagleB200UpdateTransitionMatrices(h_, e, p, d1, d2, t, n);
    }
    int updateTransitionMatricesWithModelCategories(int* e, const int* p, const int* d1,
                                                    const int* d2, const double* t,
                                                    int n) override {
        return beagleB200UpdateTransitionMatricesWithModelCategories(h_, e, p, d1, d2, t, n);
    }
    int updateTransitionMatricesWithMultipleModels(const int* e, const int* r, const int* p,
                                                   const int* d1, const int* d2, const double* t,
                                                   int n) override {
        return beagleB200UpdateTransitionMatricesWithMultipleModels(h_, e, r, p, d1, d2, t, n);
    }
    // The dispatcher hands operations over as flat int arrays
    // (libhmsbeagle/beagle.cpp, beagleUpdatePartials); seven ints per op.
    int updatePartials(const int* ops, int n, int cum) override {
        return beagleB200UpdatePartials(h_, reinterpret_cast<const BeagleB200Operation*>(ops), n,
                                        cum);
    }
    int updatePrePartials(const int* ops, int n, int cum) override {
        return beagleB200UpdatePrePartials(h_, reinterpret_cast<const BeagleB200Operation*>(ops),
                                           n, cum);
    }
    int updatePartialsByPartition(const int* ops, int n) override {
        return beagleB200UpdatePartialsByPartition(
            h_, reinterpret_cast<const BeagleB200OperationByPartition*>(ops), n);
    }
    int updatePrePartialsByPartition(const int* ops, int n) override {
        return beagleB200UpdatePrePartialsByPartition(
            h_, reinterpret_cast<const BeagleB200OperationByPartition*>(ops), n);
    }
    int waitForPartials(const int* d, int n) override { return beagleB200WaitForPartials(h_, d, n); }
    int accumulateScaleFactors(const int* s, int n, int cum) override {
        return beagleB200AccumulateScaleFactors(h_, s, n, cum);
    }
    int accumulateScaleFactorsByPartition(const int* s, int n, int cum, int part) override {
        return beagleB200AccumulateScaleFactorsByPartition(h_, s, n, cum, part);
    }
    int removeScaleFactors(const int* s, int n, int cum) override {
        return beagleB200RemoveScaleFactors(h_, s, n, cum);
    }
    int removeScaleFactorsByPartition(const int* s, int n, int cum, int part) override {
        return beagleB200RemoveScaleFactorsByPartition(h_, s, n, cum, part);
    }
    int resetScaleFactors(int cum) override { return beagleB200ResetScaleFactors(h_, cum); }
    int resetScaleFactorsByPartition(int cum, int part) override {
        return beagleB200ResetScaleFactorsByPartition(h_, cum, part);
    }
    int copyScaleFactors(int d, int s) override { return beagleB200CopyScaleFactors(h_, d, s); }
    int getScaleFactors(int s, double* out) override {
        return beagleB200GetScaleFactors(h_, s, out);
    }
    int calculateRootLogLikelihoods(const int* b, const int* w, const int* f, const int* s,
                                    int n, double* out) override {
        return beagleB200CalculateRootLogLikelihoods(h_, b, w, f, s, n, out);
    }
    int calculateRootLogLikelihoodsByPartition(const int* b, const int* w, const int* f,
                                               const int* s, const int* parts, int nparts, int n,
                                               double* byPart, double* out) override {
        return beagleB200CalculateRootLogLikelihoodsByPartition(h_, b, w, f, s, parts, nparts, n,
                                                                byPart, out);
    }
    // Rates and cumulative scale indices are not needed: D carries r_c, and
    // the scale factors cancel in the num / den ratio.
    int calculateEdgeDerivatives(const int* post, const int* pre, const int* dmat,
                                 const int* w, const int* /*rates*/, const int* /*cum*/, int n,
                                 double* site, double* sum, double* sumsq) override {
        return beagleB200CalculateEdgeDerivatives(h_, post, pre, dmat, w, n, site, sum, sumsq);
    }
    int calculateCrossProducts(const int* post, const int* pre, const int* rates, const int* w,
                               const double* t, int n, double* sum, double* sumsq) override {
        return beagleB200CalculateCrossProductDerivative(h_, post, pre, rates, w, t, n, sum,
                                                         sumsq);
    }
    int calculateEdgeLogLikelihoods(const int* pa, const int* ch, const int* p, const int* d1,
                                    const int* d2, const int* w, const int* f, const int* s,
                                    int n, double* lnl, double* o1, double* o2) override {
        return beagleB200CalculateEdgeLogLikelihoods(h_, pa, ch, p, d1, d2, w, f, s, n, lnl, o1,
                                                     o2);
    }
    int calculateEdgeLogLikelihoodsByPartition(const int* pa, const int* ch, const int* p,
                                               const int* d1, const int* d2, const int* w,
                                               const int* f, const int* s, const int* parts,
                                               int np, int n, double* byp, double* lnl,
                                               double* d1byp, double* o1, double* d2byp,
                                               double* o2) override {
        return beagleB200CalculateEdgeLogLikelihoodsByPartition(h_, pa, ch, p, d1, d2, w, f, s,
                                                                parts, np, n, byp, lnl, d1byp,
                                                                o1, d2byp, o2);
    }
    int getLogLikelihood(double* out) override { return beagleB200GetLogLikelihood(h_, out); }
    int getDerivatives(double* d1, double* d2) override {
        return beagleB200GetDerivatives(h_, d1, d2);
    }
    int getSiteLogLikelihoods(double* out) override {
        return beagleB200GetSiteLogLikelihoods(h_, out);
    }
    int getSiteDerivatives(double* d1, double* d2) override {
        return beagleB200GetSiteDerivatives(h_, d1, d2);
    }

private:
    long precision_;
    int h_ = -1;
    long flags_ = 0;
    char* impl_name_ = nullptr;
};

class B200ImplFactory final : public beagle::BeagleImplFactory {
public:
    B200ImplFactory(long precision, long resourceFlags)
        : precision_(precision),
          flags_((resourceFlags & ~(BEAGLE_FLAG_PRECISION_SINGLE | BEAGLE_FLAG_PRECISION_DOUBLE)) |
                 precision) {}

    beagle::BeagleImpl* createImpl(int tipCount, int partialsBufferCount, int compactBufferCount,
                                   int stateCount, int patternCount, int eigenBufferCount,
                                   int matrixBufferCount, int categoryCount, int scaleBufferCount,
                                   int resource, int pluginResource, long preferenceFlags,
                                   long requirementFlags, int* errorCode) override {
        B200Impl* impl = new (std::nothrow) B200Impl(precision_);
        if (!impl) {
            *errorCode = BEAGLE_ERROR_OUT_OF_MEMORY;
            return nullptr;
        }
        const int rc = impl->createInstance(
            tipCount, partialsBufferCount, compactBufferCount, stateCount, patternCount,
            eigenBufferCount, matrixBufferCount, categoryCount, scaleBufferCount, resource,
            pluginResource, preferenceFlags, requirementFlags);
        if (rc != BEAGLE_SUCCESS) {
            delete impl;
            *errorCode = rc;
            return nullptr;
        }
        *errorCode = BEAGLE_SUCCESS;
        return impl;
    }

    const char* getName() override {
        return precision_ == BEAGLE_FLAG_PRECISION_DOUBLE ? "B200-sm100a-Double"
                                                          : "B200-sm100a-Mixed";
    }
    const long getFlags() override { return flags_; }

private:
    long precision_;
    long flags_;
};

// Resources: one per CUDA device, as beagleB200GetResourceList lists them
// (pluginResourceNumber = device ordinal).  Factories are offered only when
// some device is usable, like CUDAPlugin.cpp does for CUDA devices.
class B200Plugin : public beagle::plugin::Plugin {
public:
    B200Plugin() : Plugin("GPU-B200", "GPU-CUDA") {
        BeagleB200ResourceList* rl = beagleB200GetResourceList();
        long any = 0;
        for (int k = 0; rl && k < rl->length; ++k) {
            BeagleResource r;
            r.name = rl->list[k].name;
            r.description = rl->list[k].description;
            r.supportFlags = rl->list[k].supportFlags;
            r.requiredFlags = rl->list[k].requiredFlags;
            beagleResources.push_back(r);
            any |= r.supportFlags;
        }
        if (any) {
            for (long prec : {BEAGLE_FLAG_PRECISION_DOUBLE, BEAGLE_FLAG_PRECISION_SINGLE}) {
                own_.push_back(new B200ImplFactory(prec, any));
                beagleFactories.push_back(own_.back());
            }
        }
    }
    // The dispatcher keeps its plugins for the life of the process and never
    // destroys them through this type; deleting through the derived type
    // avoids the factories' non-virtual base destructor.
    ~B200Plugin() {
        for (B200ImplFactory* f : own_) delete f;
    }

private:
    std::vector<B200ImplFactory*> own_;
};

}  // namespace b200plugin

extern "C" {
__attribute__((visibility("default"))) void* plugin_init(void) {
    return new b200plugin::B200Plugin();
}
}
