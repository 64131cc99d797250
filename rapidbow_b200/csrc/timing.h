// Optional per-kernel CUDA-event timing of the library's own launches (off by default).  When
// enabled, every timed launch is bracketed by two events recorded on its stream; no host
// synchronisation is added.  Totals are read back after the caller has synchronised.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace rbw {

enum TimedKernel : uint32_t {
    kTimedLookupPass = 0,   // tensor-core lookup pass (lookupPassTc)
    kTimedLookupSimt = 1,   // FP32 SIMT lookup
    kTimedRegroup = 2,      // scan + tile list + scatter between lookup passes
    kTimedAssign = 3,       // k-means assign
    kTimedUpdate = 4,       // k-means update
    kTimedScore = 5,        // inverted-file scoring (query preparation, scoring, merge)
    kTimedIndex = 6,        // inverted-file construction
    kTimedScorePrep = 7,    // query preparation alone (inside kTimedScore)
    kTimedScoreMerge = 8,   // merge of the per-CTA candidates alone (inside kTimedScore)
    kTimedCount = 9,
};

bool timingEnabled();
void timingEnable(bool on);
void timingReset();
// Sums the elapsed time of all completed launches of `k` (events must have completed).
void timingRead(TimedKernel k, double* totalMs, uint64_t* launches);

class ScopedKernelTimer
{
public:
    ScopedKernelTimer(TimedKernel k, cudaStream_t s);
    ~ScopedKernelTimer();
    ScopedKernelTimer(const ScopedKernelTimer&) = delete;
    ScopedKernelTimer& operator=(const ScopedKernelTimer&) = delete;

private:
    TimedKernel mKernel;
    cudaStream_t mStream;
    cudaEvent_t mStart = nullptr;
    bool mActive = false;
};

} // namespace rbw
