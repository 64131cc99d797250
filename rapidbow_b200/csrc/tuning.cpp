#include "tuning.h"
#include "rbw_common.cuh"

#include <map>
#include <mutex>
#include <tuple>

namespace rbw {
namespace {

using Key = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>; // param, B, L, bucket
std::mutex gMu;
std::map<Key, uint32_t> gTable;

bool valid(TuneParam p, uint32_t v)
{
    switch (p) {
    case kTuneAssignCtasPerSm: return v >= 1 && v <= 8;
    case kTuneAssignFCtasPerSm: return v >= 1 && v <= 3;
    case kTuneScatterRows: return v == 8 || v == 16 || v == 32;
    case kTuneDbShardTables: return v == 1 || v == 2;
    case kTuneLookupSchedule: return v == 1 || v == 2;
    case kTuneAssignSums: return v == 1 || v == 2;
    default: return false;
    }
}

} // namespace

uint32_t tuneBucket(uint64_t n)
{
    uint32_t b = 0;
    while (n > 1) {
        n >>= 1;
        b++;
    }
    return b;
}

uint32_t tuneDefault(TuneParam p)
{
    switch (p) {
    case kTuneAssignCtasPerSm: return 6;
    case kTuneAssignFCtasPerSm: return 3;
    case kTuneScatterRows: return 16;
    case kTuneDbShardTables: return 1;
    case kTuneLookupSchedule: return 1;
    case kTuneAssignSums: return 1;
    default: return 0;
    }
}

uint32_t tunedValue(TuneParam p, uint32_t B, uint32_t L, uint64_t n)
{
    const uint32_t bucket = tuneBucket(n);
    std::lock_guard<std::mutex> lk(gMu);
    auto it = gTable.find(Key{p, B, L, bucket});
    if (it == gTable.end() && L != 0) it = gTable.find(Key{p, B, 0u, bucket});
    return it == gTable.end() ? tuneDefault(p) : it->second;
}

void setTunedValue(TuneParam p, uint32_t B, uint32_t L, uint32_t bucket, uint32_t value)
{
    if (p >= kTuneParamCount) throw Error(kInvalidArg, "unknown tuning parameter");
    if (B < 2 || B > kMaxBranch || bucket > 63) throw Error(kInvalidArg, "bad tuning key");
    std::lock_guard<std::mutex> lk(gMu);
    if (value == 0) {
        gTable.erase(Key{p, B, L, bucket});
        return;
    }
    if (!valid(p, value)) throw Error(kInvalidArg, "value out of range for this tuning parameter");
    gTable[Key{p, B, L, bucket}] = value;
}

void clearTuning()
{
    std::lock_guard<std::mutex> lk(gMu);
    gTable.clear();
}

} // namespace rbw
