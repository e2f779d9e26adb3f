// Root log-likelihood on caller-owned device buffers, with no allocation.
//
// Some callers cannot let a library call cudaMalloc.  One example is a
// framework that owns every byte of device memory through its own allocator
// (a caching allocator, a memory pool, an arena sized up front).  Another is a
// real-time loop in which cudaMalloc's implicit device synchronisation is not
// acceptable.  For them, beagleB200RootLogLikelihoodsNoAlloc computes the
// pattern-weighted root log-likelihood into buffers the caller passes in.  The
// only scratch it needs, the per-block partial sums of the two-pass FP64
// reduction, lives in the file-scope device array below: a fixed
// 64 KiB (8192 doubles) on every GPU that loads the library, held until the
// process exits.
//
// The array is shared by every call on a device and keeps the previous call's
// contents.  Nothing needs clearing: each call writes every slot it later
// reads (one partial per pattern block) before reading it.  Two calls that
// overlap on the GPU (different streams, or different host threads on the
// same device) race on the array; callers must order them.
#include <cstdint>

#include "b200_kernels.h"
#include "beagle_b200.h"

namespace b200 {
namespace {

constexpr int kScratchDoubles = 8192;   // 64 KiB: one double per 128-pattern block
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// The array's device address on the current device.  In host code the symbol
// g_noalloc_scratch is a host-side stand-in, not a device address.  The
// address is looked up on every call rather than cached, so that it is the
// current context's even after a cudaDeviceReset or under another primary
// context.  The lookup is cheap once the module is loaded; the first call on
// a device may load it, which is why that call must come before any stream
// capture.
cudaError_t scratch_address(double** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    *out = static_cast<double*>(p);
    return e;
}

bool aligned(const void* p, std::uintptr_t a) {
    return (reinterpret_cast<std::uintptr_t>(p) % a) == 0;
}

}  // namespace
}  // namespace b200

extern "C" int beagleB200RootLogLikelihoodsNoAlloc(
    int device, void* stream, const void* rootPartials, int doublePrecision, int stateCount,
    int patternCount, int categoryCount, const double* categoryWeights,
    const double* stateFrequencies, const double* cumulativeScaleFactors,
    const double* patternWeights, double* outSiteLogLikelihoods, double* outSumLogLikelihood) {
    if (!rootPartials || !categoryWeights || !stateFrequencies || !patternWeights ||
        !outSiteLogLikelihoods || !outSumLogLikelihood)
        return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    if (stateCount < 2 || stateCount > 64 || categoryCount < 1 || patternCount < 1)
        return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    // Partials rows are read as 16-byte vectors; the FP64 arrays as doubles.
    // A misaligned pointer (an offset view into a larger allocation) is
    // refused here, before anything is queued.
    if (!b200::aligned(rootPartials, 16) || !b200::aligned(categoryWeights, 8) ||
        !b200::aligned(stateFrequencies, 8) || !b200::aligned(patternWeights, 8) ||
        !b200::aligned(cumulativeScaleFactors, 8) || !b200::aligned(outSiteLogLikelihoods, 8) ||
        !b200::aligned(outSumLogLikelihood, 8))
        return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    // One scratch double per 128-pattern block: at most 8192 * 128 patterns.
    if (b200::reduction_blocks(patternCount) > b200::kScratchDoubles)
        return BEAGLE_B200_ERROR_OUT_OF_RANGE;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        (void)cudaGetLastError();
        return BEAGLE_B200_ERROR_NO_RESOURCE;
    }
    double* scratch = nullptr;
    cudaError_t e = b200::scratch_address(&scratch);
    if (e == cudaSuccess) {
        b200::Dims d;
        d.S = stateCount;
        d.Sg = (stateCount + 3) / 4 * 4;
        d.P = patternCount;
        d.Pp = patternCount;
        d.C = categoryCount;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        e = doublePrecision
                ? b200::launch_root_lnl<double>(rootPartials, categoryWeights, stateFrequencies,
                                                cumulativeScaleFactors, patternWeights, d,
                                                outSiteLogLikelihoods, scratch,
                                                outSumLogLikelihood, s, false)
                : b200::launch_root_lnl<float>(rootPartials, categoryWeights, stateFrequencies,
                                               cumulativeScaleFactors, patternWeights, d,
                                               outSiteLogLikelihoods, scratch,
                                               outSumLogLikelihood, s, false);
    }
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return BEAGLE_B200_ERROR_GENERAL;
    }
    return BEAGLE_B200_SUCCESS;
}
