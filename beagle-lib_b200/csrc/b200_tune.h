// Kernel-variant autotuner.  Several launches have more than one kernel shape
// that computes the same result (patterns per thread, thread per pattern vs
// thread per category); which is fastest depends on the pattern count, the
// category count and the length of the op list.  The first call of a given
// shape times every variant on the caller's stream with CUDA events and
// caches the fastest for the life of the process.
//
// Only idempotent launches are tuned (a post-order list that adds into a
// cumulative scale buffer, or that reads a buffer it writes later, is not):
// each candidate writes the same outputs, and the winner runs once more for
// the caller's result.  A stream that is being captured into a CUDA graph is
// never tuned; it gets the cached choice or the default.
//
// Environment:
//   BEAGLE_B200_TUNE=0            no tuning, always the default variant;
//   BEAGLE_B200_FORCE_VARIANT=v   always variant v (clamped to the range),
//                                 used by the parity tests to cover each one;
//                                 "a,b,c" pins post-order walk, pre-order walk
//                                 and derivative separately (-1 = tune);
//   BEAGLE_B200_TUNE_LOG=1        print each candidate's time to stderr.
#pragma once
#include <cuda_runtime.h>
#include <functional>

namespace b200 {

enum TuneKind { kTuneWalkPost = 1, kTuneWalkPre = 2, kTuneDeriv = 3, kTuneFused = 4 };

struct TuneKey {
    int kind, dbl, C, Pp, count_class, device;
};

// Variant to pass to the launcher: the cached or measured fastest of
// `nvariants`, or -1 for the launcher's default.  `run(v)` enqueues variant v
// on `s` and returns its launch status.  With `may_time` false nothing runs.
int tune_pick(const TuneKey& key, int nvariants, bool may_time, cudaStream_t s,
              const std::function<cudaError_t(int)>& run);

// Bucket of a list length for TuneKey::count_class (powers of two).
int tune_count_class(int n);

}  // namespace b200
