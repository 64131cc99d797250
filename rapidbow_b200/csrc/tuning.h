// Launch parameters chosen by the host's autotuner (rapidbow_b200/autotune.py), kept per
// (parameter, branch factor, tree levels, descriptor-count bucket).  A kernel launcher asks for
// its value with the shape of its workload; unset entries give the built-in default.
#pragma once
#include <cstdint>

namespace rbw {

enum TuneParam : uint32_t {
    kTuneAssignCtasPerSm = 0,  // uint8 k-means assign: resident CTAs per SM, 1..8 (default 6)
    kTuneAssignFCtasPerSm = 1, // float-center assign: resident CTAs per SM, 1..3 (default 3)
    kTuneScatterRows = 2,      // lookup regroup scatter: rows per thread, 8 | 16 | 32 (default 16)
    kTuneDbShardTables = 3,    // inverted file: 1 one CSR per 2,560-document shard while small (default), 2 one CSR
    kTuneLookupSchedule = 4,   // tensor-core lookup of RBW_LOOKUP_AUTO: 1 pair schedule (default), 2 ring
    kTuneAssignSums = 5,       // uint8 k-means center sums: 1 shared atomics (default), 2 tensor core
    kTuneParamCount = 6,
};

// floor(log2(max(n, 1))): workloads within a factor of two share an entry.
uint32_t tuneBucket(uint64_t n);
// The value for a workload of n descriptors (L = 0 matches entries stored for any depth).
uint32_t tunedValue(TuneParam p, uint32_t B, uint32_t L, uint64_t n);
uint32_t tuneDefault(TuneParam p);
// Throws kInvalidArg for a value the parameter cannot take; value 0 removes the entry.
void setTunedValue(TuneParam p, uint32_t B, uint32_t L, uint32_t bucket, uint32_t value);
void clearTuning();

} // namespace rbw
