// Device-resident inverted file and hierarchical tf-idf scoring (reference: DataBase.cpp:39-197).
//
// Documents (DataBase.cpp:39-69):
//   * addDoc only stages the host leaf indices; the device work happens at the next query, for
//     the documents staged since the last one;
//   * docPrepKernel, one CTA per new document: sorts its leaf words in shared memory, computes
//     the L1 norm of its weight vector over all levels in the reference's order (levels
//     leaf->root, descriptors in ascending leaf order, double sum; DataBase.cpp:54-68) and
//     run-length encodes it into (leaf, tf) pairs kept per document.
// Inverted file, in two segments, each a CSR over leaves of (slot, d) pairs, where
// d = float(tf) * w_leaf * rcp is the document's leaf-level entry (DataBase.cpp:129, the same
// float products the query would form), plus the raw tf per pair for the upper levels:
//   * main: documents [0, mainEnd), rebuilt when the newer documents outgrow a fraction of it;
//   * delta: documents [mainEnd, n), rebuilt from those documents alone after every add, so an
//     add costs work in proportion to the delta, not to the database.
//   A leaf's pairs over both segments are the reference's sorted posting list with repeated
//   document ids folded into tf.  Subtree posting counts of every word (with multiplicity,
//   both segments) drive the reference's level skip rule: a non-leaf word is scored only if
//   its subtree holds < 16 + 4k postings (DataBase.h:60-61, DataBase.cpp:125).
// Queries (any number per launch, uneven sizes):
//   * queryPrepKernel, one CTA per query: sort, query L1 norm (same order as documents), and
//     the (level, word, run) entries that survive the skip rule;
//   * scoreKernel, one CTA per query: warps take entries and add, for every document in the
//     entry's postings, the reference's term |q - d| - (q + d), q = run*w*qRcp and
//     d = tf*w*dRcp in float (DataBase.cpp:117,127-131; d read from the pair at the leaf
//     level, formed from the summed tf at upper levels).  Each document's terms are summed in
//     64-bit fixed point (2^-56 units), so the sum does not depend on the order in which warps
//     add them; the score is float(sum + 2) (DataBase.cpp:170-174); the k best are chosen by a
//     radix select on (score, document id).
// Ordering: index updates run on the database's own stream; a query stream waits for the last
// update (event), and an update first waits for the queries launched since the previous one,
// so no host synchronisation is needed between adds and batched queries.
#include "capi_internal.h"
#include "kmeans.cuh"
#include "timing.h"
#include "tuning.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <optional>
#include <shared_mutex>
#include <unordered_map>
#include <vector>

namespace rbw {
namespace {

constexpr uint32_t kMaxDocDesc = 32768;   // descriptors sorted in shared memory; larger ones in global memory
constexpr uint32_t kPrepThreads = 512;
constexpr uint32_t kScoreThreads = 1024;
constexpr uint32_t kFlatList = 256;        // leaf lists shorter than this are walked flattened per warp batch
constexpr uint32_t kFlatDepth = 8;         // pairs per lane in flight in the flattened walk
constexpr uint32_t kSegThreads = 256;
constexpr uint32_t kSmemDocs = 20480;     // per-document accumulators kept in shared memory
constexpr uint32_t kShardDocs = 2560;     // documents per inverted-file shard
constexpr uint32_t kGroupShards = kSmemDocs / kShardDocs; // shards per group of kSmemDocs documents (8)
constexpr uint64_t kShardTableMinBytes = 64ull << 20; // per-shard CSR tables always allowed up to this size
constexpr uint32_t kMaxK = 1024;          // results selected in shared memory; more in global memory
constexpr double kFixScale = 72057594037927936.0; // 2^56
constexpr uint32_t kDeltaMinDocs = 256;   // the delta may always hold this many documents
constexpr uint32_t kDeltaFraction = 4;    // ... or up to main / kDeltaFraction

struct Entry {
    uint32_t level;
    uint32_t word;   // index of the word within its level (= node index at level + 1)
    uint32_t run;    // query descriptors under this word
    uint32_t widx;   // index into the weight table: levelBeg(level) * B + word
};

__host__ __device__ inline uint64_t levelBegDev(uint32_t B, uint32_t level)
{
    uint64_t acc = 0;
    for (uint32_t i = 0; i < level; i++) acc = acc * B + 1;
    return acc;
}

__host__ __device__ inline uint64_t ipowDev(uint32_t b, uint32_t e)
{
    uint64_t r = 1;
    for (uint32_t i = 0; i < e; i++) r *= b;
    return r;
}

uint32_t nextPow2(uint32_t n)
{
    uint32_t p = 1;
    while (p < n) p <<= 1;
    return p;
}

uint32_t blocks(uint64_t n, uint32_t t) { return static_cast<uint32_t>((n + t - 1) / t); }

// Ascending bitonic sort of nPow2 keys in shared memory (all threads of the CTA take part).
template <typename T>
__device__ void bitonicSortShared(T* keys, uint32_t nPow2)
{
    for (uint32_t k = 2; k <= nPow2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            // pair t compares i = (t with a zero bit inserted at j) with i + j
            for (uint32_t t = threadIdx.x; t < nPow2 / 2; t += blockDim.x) {
                const uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                const uint32_t ixj = i | j;
                const bool up = (i & k) == 0;
                const T a = keys[i], b = keys[ixj];
                if ((a > b) == up) {
                    keys[i] = b;
                    keys[ixj] = a;
                }
            }
            __syncthreads();
        }
    }
}

// Warp-aggregated slot allocation: the warp's lanes with `take` get consecutive slots from
// *counter (one atomic per warp).  Every lane of the warp must call it.
__device__ __forceinline__ uint32_t warpSlot(bool take, uint32_t* counter)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t mask = __ballot_sync(0xFFFFFFFFu, take);
    uint32_t base = 0;
    if (lane == 0 && mask != 0) base = atomicAdd(counter, uint32_t(__popc(mask)));
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// Loads n leaf indices, sorts them and returns how many are valid (< nbLeaves): leaves out of
// range sort to the end and are ignored, so a bad index never reaches a table lookup.
__device__ uint32_t loadAndSort(const uint32_t* src, uint32_t n, uint32_t* keys, uint64_t nbLeaves, uint32_t* nValid)
{
    uint32_t nPow2 = 1;
    while (nPow2 < n) nPow2 <<= 1;
    if (threadIdx.x == 0) *nValid = 0;
    __syncthreads();
    uint32_t mine = 0;
    for (uint32_t i = threadIdx.x; i < nPow2; i += blockDim.x) {
        const uint32_t v = i < n ? src[i] : 0xFFFFFFFFu;
        keys[i] = v;
        mine += v < nbLeaves ? 1u : 0u;
    }
    atomicAdd(nValid, mine);
    __syncthreads();
    bitonicSortShared(keys, nPow2);
    return *nValid;
}

// Double sum of the weights of every (level, descriptor) in the reference's order (levels
// leaf->root, descriptors in ascending leaf order).  Warp-collective: the lanes gather 32
// weights at a time (the next 32 in flight while the current ones are added) and every lane
// adds them one after another in the same order, so all lanes hold the same sum.
__device__ double l1NormWarp(const uint32_t* sorted, uint32_t n, const float* weights, uint32_t B, uint32_t L)
{
    const uint32_t lane = threadIdx.x & 31u;
    double norm = 0;
    uint32_t span = 1; // B^it; leaf indices are 32-bit, so is every span
    for (uint32_t it = 0; it < L; it++) {
        const float* lw = weights + levelBegDev(B, L - 1 - it) * B;
        float next = lane < n ? lw[sorted[lane] / span] : 0.f;
        for (uint32_t base = 0; base < n; base += 32) {
            const float cur = next;
            const uint32_t ahead = base + 32 + lane;
            next = ahead < n ? lw[sorted[ahead] / span] : 0.f;
            // all 32 shuffles first, so only the additions form the dependent chain
            float t[32];
#pragma unroll
            for (uint32_t j = 0; j < 32; j++) t[j] = __shfl_sync(0xFFFFFFFFu, cur, j);
            if (n - base >= 32) {
#pragma unroll
                for (uint32_t j = 0; j < 32; j++) norm += t[j];
            } else {
#pragma unroll
                for (uint32_t j = 0; j < 32; j++)
                    if (j < n - base) norm += t[j];
            }
        }
        span *= B;
    }
    return norm;
}

// The same sum by the whole block, when it can be shown that no addition of the reference's
// order rounds in a way that matters.  Every term must be finite and >= 0.  Terms below 2^-70
// ("tiny": the idf weights clamped to FLT_MIN for words in more documents than the vocabulary
// was built for, Vocabulary.cpp:103-108) are set aside; every other term is an integer multiple
// of 2^e, e = the lowest set bit of any of them.
//   * If the exact total of those terms is below 2^(e + 53), each of their partial sums is an
//     exactly representable double.
//   * If all tiny terms together stay below 2^(m - 53), m = the exponent of the smallest other
//     term, then every tiny term, and whatever tiny terms sum to before the first other term,
//     is less than half an ulp of the running sum it meets (which is at least that smallest
//     term), so it rounds away.
// Together: the in-order double sum equals the exact total of the other terms, which the block
// forms here in any order with 64-bit integers (one pass for the bounds, one for the total).
// Call from every thread.  Returns false when this cannot be shown; the caller then adds the
// terms in order (l1NormWarp) in one warp while the others go on.
__device__ bool l1NormBlockExact(const uint32_t* sorted, uint32_t n, const float* weights, uint32_t B, uint32_t L,
                                 double* norm)
{
    constexpr uint32_t kTinyBits = uint32_t(127 - 70) << 23; // float bits of 2^-70
    __shared__ int32_t sLsb;
    __shared__ uint32_t sBad, sMinBig, sMaxTiny, sTiny;
    __shared__ unsigned long long sTotal;
    if (threadIdx.x == 0) {
        sLsb = 0x7FFFFFFF;
        sBad = 0;
        sMinBig = 0xFFFFFFFFu;
        sMaxTiny = 0;
        sTiny = 0;
        sTotal = 0;
    }
    __syncthreads();
    // exponent of bit 0 of the significand and the significand (implicit bit included)
    auto split = [](uint32_t bits, int32_t& e0, uint32_t& m) {
        const uint32_t ef = (bits >> 23) & 0xFFu;
        m = (bits & 0x7FFFFFu) | (ef ? 0x800000u : 0u);
        e0 = int32_t(ef ? ef : 1u) - 150;
    };
    int32_t lsb = 0x7FFFFFFF;
    uint32_t bad = 0, minBig = 0xFFFFFFFFu, maxTiny = 0, tiny = 0;
    uint32_t span = 1;
    for (uint32_t it = 0; it < L; it++) {
        const float* lw = weights + levelBegDev(B, L - 1 - it) * B;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t bits = __float_as_uint(lw[sorted[i] / span]);
            if ((bits & 0x7FFFFFFFu) == 0) continue; // +-0 adds nothing
            if ((bits >> 31) != 0 || ((bits >> 23) & 0xFFu) == 0xFFu) {
                bad = 1;                              // negative, infinite or NaN
                continue;
            }
            if (bits < kTinyBits) {                   // positive floats order like their bits
                tiny++;
                maxTiny = max(maxTiny, bits);
                continue;
            }
            minBig = min(minBig, bits);
            int32_t e0;
            uint32_t m;
            split(bits, e0, m);
            lsb = min(lsb, e0 + int32_t(__ffs(m)) - 1);
        }
        span *= B;
    }
    atomicMin(&sLsb, lsb);
    if (bad) atomicOr(&sBad, 1u);
    if (tiny) {
        atomicAdd(&sTiny, tiny);
        atomicMax(&sMaxTiny, maxTiny);
    }
    atomicMin(&sMinBig, minBig);
    __syncthreads();
    const int32_t e = sLsb;
    bool ok = !sBad;
    if (ok && sTiny) {
        // all tiny terms < sTiny * 2^(exp(maxTiny) + 1) <= 2^(ceil(log2 sTiny) + exp(maxTiny) + 1);
        // one more factor of two covers the rounding of their own in-order sum
        const int32_t expTiny = int32_t((sMaxTiny >> 23) & 0xFFu) - 127;
        const int32_t logCount = 32 - int32_t(__clz(sTiny - 1u)); // ceil(log2(sTiny)), 0 for 1
        const int32_t expBig = int32_t((sMinBig >> 23) & 0xFFu) - 127;
        ok = sMinBig != 0xFFFFFFFFu && logCount + expTiny + 2 <= expBig - 53;
    }
    if (!ok) return false;
    if (e == 0x7FFFFFFF) {
        *norm = 0.0; // no term above the tiny ones (and none of those)
        return sTiny == 0;
    }
    constexpr unsigned long long kLimit = 1ull << 53;
    unsigned long long total = 0;
    span = 1;
    for (uint32_t it = 0; it < L && !bad; it++) {
        const float* lw = weights + levelBegDev(B, L - 1 - it) * B;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t bits = __float_as_uint(lw[sorted[i] / span]);
            if ((bits & 0x7FFFFFFFu) == 0 || bits < kTinyBits) continue;
            int32_t e0;
            uint32_t m;
            split(bits, e0, m);
            const int32_t tz = __ffs(m) - 1;
            m >>= tz;                          // odd significand, lowest set bit 2^(e0 + tz)
            const int32_t shift = e0 + tz - e; // >= 0: e is the lowest of those bits
            if (shift + 32 - int32_t(__clz(m)) > 53) {
                bad = 1;                       // the term alone reaches 2^(e + 53)
                break;
            }
            total += static_cast<unsigned long long>(m) << shift;
            if (total >= kLimit) {
                bad = 1;
                break;
            }
        }
        span *= B;
    }
    if (bad) atomicOr(&sBad, 1u);
    atomicAdd(&sTotal, total); // < blockDim * 2^53: no overflow
    __syncthreads();
    if (sBad || sTotal >= kLimit) return false;
    *norm = ldexp(static_cast<double>(sTotal), e);
    return true;
}

// ------------------------------------------------------------------ documents
// One CTA per new document.  newLeaves holds the new documents' leaves back to back, starting at
// posting offset docOff[s0].  Without gkeys, CTA i prepares slot s0 + i in shared memory and
// skips documents above kMaxDocDesc descriptors; with gkeys, CTA i prepares slot slotList[i],
// sorting in its gstride-word slice of gkeys.
__global__ void __launch_bounds__(kPrepThreads) docPrepKernel(const uint32_t* newLeaves, const uint64_t* docOff,
                                                              uint32_t s0, const uint32_t* slotList, uint32_t* gkeys,
                                                              uint32_t gstride, const float* weights, uint32_t B,
                                                              uint32_t L, uint64_t nbLeaves, float* rcpF,
                                                              uint64_t* docPairs, uint32_t* pairCount)
{
    extern __shared__ uint32_t skeys[];
    __shared__ uint32_t cnt, nValid;
    const uint32_t slot = gkeys ? slotList[blockIdx.x] : s0 + blockIdx.x;
    const uint64_t beg = docOff[slot];
    const uint32_t nAll = static_cast<uint32_t>(docOff[slot + 1] - beg);
    if (gkeys == nullptr && nAll > kMaxDocDesc) return; // prepared by the global-memory launch
    uint32_t* keys = gkeys ? gkeys + uint64_t(blockIdx.x) * gstride : skeys;
    if (threadIdx.x == 0) cnt = 0;
    const uint32_t n = loadAndSort(newLeaves + (beg - docOff[s0]), nAll, keys, nbLeaves, &nValid);
    double norm = 0;
    if (l1NormBlockExact(keys, n, weights, B, L, &norm)) {
        if (threadIdx.x == 0) rcpF[slot] = float(1 / norm); // DataBase.cpp:68
    } else if (threadIdx.x < 32) {
        norm = l1NormWarp(keys, n, weights, B, L);
        if (threadIdx.x == 0) rcpF[slot] = float(1 / norm);
    }
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t k = i < n ? keys[i] : 0u;
        const bool head = i < n && (i == 0 || keys[i - 1] != k);
        const uint32_t pos = warpSlot(head, &cnt);
        if (head) {
            uint32_t run = 1;
            while (i + run < n && keys[i + run] == k) run++;
            docPairs[beg + pos] = (uint64_t(k) << 32) | run;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) pairCount[slot] = cnt;
}

// Offset-table index of (document slot, leaf) in a segment.  Grouped layout: groups of
// kSmemDocs documents, then leaves, then the group's kGroupShards shards of kShardDocs
// documents, so any aligned run of shards of a group holds one leaf's pairs in one range, and a
// whole group one range per run of leaves.  Single layout (grouped = false): one CSR by leaf.
__host__ __device__ __forceinline__ uint64_t segIndex(uint32_t slot, uint64_t leaf, uint32_t groupBeg,
                                                      uint64_t nbLeaves, bool grouped)
{
    if (!grouped) return leaf;
    return ((uint64_t(slot / kSmemDocs - groupBeg) * nbLeaves + leaf) * kGroupShards) +
           (slot % kSmemDocs) / kShardDocs;
}

// Per-table-entry pair counts and per-leaf posting counts of the documents [s0, s0 + gridDim.x).
__global__ void segCountKernel(const uint64_t* docOff, const uint64_t* docPairs, const uint32_t* pairCount,
                               uint32_t s0, uint32_t groupBeg, uint64_t nbLeaves, bool grouped,
                               uint32_t* leafPairCnt, unsigned long long* leafPost)
{
    const uint32_t slot = s0 + blockIdx.x;
    const uint64_t beg = docOff[slot];
    for (uint32_t p = threadIdx.x; p < pairCount[slot]; p += blockDim.x) {
        const uint64_t v = docPairs[beg + p];
        const uint32_t leaf = static_cast<uint32_t>(v >> 32);
        atomicAdd(&leafPairCnt[segIndex(slot, leaf, groupBeg, nbLeaves, grouped)], 1u);
        atomicAdd(&leafPost[leaf], static_cast<unsigned long long>(static_cast<uint32_t>(v)));
    }
}

// Scatters the documents' pairs into the segment: pairs[] = slot << 32 | bits of the leaf-level
// document entry d = tf * w_leaf * rcp (DataBase.cpp:129, the same float products as at query
// time), tf[] = the raw count for the virtual inverted files of upper levels.
__global__ void segScatterKernel(const uint64_t* docOff, const uint64_t* docPairs, const uint32_t* pairCount,
                                 uint32_t s0, uint32_t groupBeg, uint64_t nbLeaves, bool grouped,
                                 const float* leafWeights, const float* rcpF, const uint32_t* leafOff,
                                 uint32_t* cursor, uint64_t* pairs, uint32_t* tfs)
{
    const uint32_t slot = s0 + blockIdx.x;
    const uint64_t beg = docOff[slot];
    const float rcp = rcpF[slot];
    for (uint32_t p = threadIdx.x; p < pairCount[slot]; p += blockDim.x) {
        const uint64_t v = docPairs[beg + p];
        const uint32_t leaf = static_cast<uint32_t>(v >> 32);
        const uint32_t tf = static_cast<uint32_t>(v);
        const float d = float(tf) * leafWeights[leaf] * rcp;
        const uint64_t idx = segIndex(slot, leaf, groupBeg, nbLeaves, grouped);
        const uint32_t pos = leafOff[idx] + atomicAdd(&cursor[idx], 1u);
        pairs[pos] = (uint64_t(slot) << 32) | __float_as_uint(d);
        tfs[pos] = tf;
    }
}

__global__ void leafOffTail(const uint32_t* leafPairCnt, uint32_t* leafOff, uint64_t nLeaves)
{
    leafOff[nLeaves] = leafOff[nLeaves - 1] + leafPairCnt[nLeaves - 1];
}

// Leaf-level word counts = main + delta postings per leaf.
__global__ void leafPostCombine(const unsigned long long* mainPost, const unsigned long long* deltaPost,
                                unsigned long long* out, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = mainPost[i] + (deltaPost ? deltaPost[i] : 0ull);
}

// Postings under each word of `level`, from the counts of the level below (bottom-up).
__global__ void wordPostKernel(unsigned long long* wordPost, uint32_t B, uint32_t level)
{
    const uint64_t nWords = ipowDev(B, level + 1);
    const uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (w >= nWords) return;
    const unsigned long long* below = wordPost + levelBegDev(B, level + 1) * B + w * B;
    unsigned long long s = 0;
    for (uint32_t c = 0; c < B; c++) s += below[c];
    wordPost[levelBegDev(B, level) * B + w] = s;
}

// ------------------------------------------------------------------ queries
// One CTA per query: without gkeys CTA i prepares query i in shared memory (skipping queries
// above kMaxDocDesc descriptors); with gkeys CTA i prepares query qList[i] in its gstride-word
// slice of gkeys.
__global__ void __launch_bounds__(kPrepThreads) queryPrepKernel(const uint32_t* qLeaves, const uint64_t* qOff,
                                                                const uint32_t* qList, uint32_t* gkeys,
                                                                uint32_t gstride, const float* weights,
                                                                const unsigned long long* wordPost, uint32_t B,
                                                                uint32_t L, uint64_t nbLeaves, uint32_t k,
                                                                float* qRcpF, Entry* entries, uint32_t* entryCount,
                                                                unsigned long long* work)
{
    extern __shared__ uint32_t skeys[];
    __shared__ uint32_t cnt, nValid;
    __shared__ unsigned long long workSum;
    const uint32_t q = gkeys ? qList[blockIdx.x] : blockIdx.x;
    const uint64_t beg = qOff[q];
    const uint32_t nAll = static_cast<uint32_t>(qOff[q + 1] - beg);
    if (gkeys == nullptr && nAll > kMaxDocDesc) return; // prepared by the global-memory launch
    uint32_t* keys = gkeys ? gkeys + uint64_t(blockIdx.x) * gstride : skeys;
    Entry* out = entries + (beg - qOff[0]) * L;
    if (threadIdx.x == 0) {
        cnt = 0;
        workSum = 0;
    }
    const uint32_t n = loadAndSort(qLeaves + beg, nAll, keys, nbLeaves, &nValid);
    double norm = 0;
    if (l1NormBlockExact(keys, n, weights, B, L, &norm)) {
        if (threadIdx.x == 0) qRcpF[q] = float(1 / norm); // DataBase.cpp:77-94
    } else if (threadIdx.x < 32) {
        norm = l1NormWarp(keys, n, weights, B, L); // while the other warps build the entries
        if (threadIdx.x == 0) qRcpF[q] = float(1 / norm);
    }
    uint32_t span = 1; // B^it; leaf indices are 32-bit, so is every span
    const uint64_t limit = 16ull + 4ull * k; // DataBase.h:60-61, DataBase.cpp:125
    unsigned long long myWork = 0;            // postings the scoring will read
    for (uint32_t it = 0; it < L; it++) {
        const uint32_t level = L - 1 - it;
        const uint64_t base = levelBegDev(B, level) * B;
        for (uint32_t i0 = 0; i0 < n; i0 += blockDim.x) {
            const uint32_t i = i0 + threadIdx.x;
            const uint32_t word = i < n ? keys[i] / span : 0u;
            bool keep = false;
            uint32_t run = 0;
            uint64_t widx = 0;
            if (i < n && (i == 0 || keys[i - 1] / span != word)) {
                // the run of `word` ends at the first key >= (word + 1) * span (keys are sorted)
                const uint64_t end = (uint64_t(word) + 1) * span;
                uint32_t lo = i + 1, hi = n;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (keys[mid] < end) lo = mid + 1;
                    else hi = mid;
                }
                run = lo - i;
                widx = base + word;
                const unsigned long long post = wordPost[widx];
                keep = it == 0 || post < limit;
                if (keep) myWork += post + 1ull;
            }
            const uint32_t p = warpSlot(keep, &cnt);
            if (keep) out[p] = Entry{level, word, run, static_cast<uint32_t>(widx)};
        }
        span *= B;
    }
    for (uint32_t off = 16; off > 0; off >>= 1) myWork += __shfl_xor_sync(0xFFFFFFFFu, myWork, off);
    if ((threadIdx.x & 31u) == 0) atomicAdd(&workSum, myWork);
    __syncthreads();
    if (threadIdx.x == 0) {
        entryCount[q] = cnt;
        work[q] = workSum;
    }
}

constexpr uint32_t kOrderMax = 4096; // batches up to this many queries are launched by work

// order[] = the queries by descending work (ties by ascending index), so the scoring launch
// starts the longest queries first and the last wave holds the short ones.  One CTA.
__global__ void __launch_bounds__(1024) workOrderKernel(const unsigned long long* work, uint32_t nq, uint32_t* order)
{
    __shared__ unsigned long long keys[kOrderMax];
    uint32_t nPow2 = 1;
    while (nPow2 < nq) nPow2 <<= 1;
    for (uint32_t i = threadIdx.x; i < nPow2; i += blockDim.x) {
        // ascending sort of (~work << 32 | index): descending work, then ascending index
        const unsigned long long w = i < nq ? (work[i] > 0xFFFFFFFEull ? 0xFFFFFFFEull : work[i]) : 0ull;
        keys[i] = i < nq ? ((0xFFFFFFFFull - w) << 32) | i : ~0ull;
    }
    __syncthreads();
    bitonicSortShared(keys, nPow2);
    for (uint32_t i = threadIdx.x; i < nq; i += blockDim.x) order[i] = static_cast<uint32_t>(keys[i]);
}

struct SegmentView {
    const uint32_t* leafOff;   // grouped: [nGroups][nbLeaves][kGroupShards] + 1; else [nbLeaves + 1]
    const uint64_t* pairs;     // slot << 32 | float bits of the leaf-level document entry
    const uint32_t* tf;        // descriptors of the document under the leaf
    uint32_t grouped;          // layout (segIndex)
    uint32_t groupBeg, nGroups;
};

struct ScoreParams {
    const Entry* entries;
    const uint32_t* entryCount;
    const uint64_t* qOff;
    const float* qRcpF;
    const float* weights;
    SegmentView seg[2];        // main, delta
    uint32_t csrPerCta;        // shards of kShardDocs documents per CTA (grouped segments)
    uint64_t nbLeaves;
    const float* rcpF;
    const uint32_t* slotDoc;
    uint32_t nDocs;
    uint32_t shardDocs;        // documents per CTA (blockIdx.y selects the shard)
    uint32_t B;
    uint32_t L;
    uint32_t k;
    unsigned long long* cand;  // [nq][shards][k] candidate keys when there are several shards
    unsigned long long* selGlobal; // k > kMaxK: [nq][shards][selStride] selection buffers
    const uint32_t* order;     // launch order of the queries (nullptr: in index order)
    uint32_t selStride;        // power of two >= k
    uint32_t* outDocs;         // [nq][k]
    float* outScores;          // [nq][k]
    uint32_t* outCount;        // [nq]
};

__device__ __forceinline__ float termOf(float q, float d) { return fabsf(q - d) - (q + d); }

// Adds a term to a document of this CTA's shard (local index `i` < shard size).
// Terms are -2 min(q, d) <= 0.  A term that rounds to 0 (|term| < 2^-57, e.g. a word whose idf
// was clamped to FLT_MIN) is added as -1 unit instead, so that a document is touched exactly
// when its accumulator is non-zero and no separate mark is stored per pair.  The change is at
// most 2^-56 per term, far below the 2^-24 resolution of the float score near 2.
__device__ __forceinline__ void addTerm(unsigned long long* acc, uint32_t i, float term)
{
    // term * 2^56 is exact in fp32 (|term| <= 2, a power-of-two scale), so rounding it to the
    // nearest integer in fp32 gives the value llrint(double(term) * 2^56) would, without FP64
    const long long fx = __float2ll_rn(term * 0x1p56f);
    atomicAdd(&acc[i], static_cast<unsigned long long>(fx < 0 ? fx : -1ll));
}

// Float bits mapped so that unsigned order is numeric order (negative scores included).
__device__ __forceinline__ uint32_t orderedBits(float f)
{
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fromOrderedBits(uint32_t o)
{
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

// The `want` smallest of n distinct keys (~0 = no key), ascending, into sel[0, want): radix
// select of the want-th smallest key, 8 bits at a time, then a bitonic sort of the winners.
// All threads of the CTA call it; keys and sel may live in shared or global memory; selCap is a
// power of two >= want.
__device__ __forceinline__ void selectSmallest(const unsigned long long* keys, uint32_t n, uint32_t want,
                                               unsigned long long* sel, uint32_t selCap)
{
    __shared__ uint32_t hist[256];
    __shared__ unsigned long long prefix;
    __shared__ uint32_t need, nSel;
    if (threadIdx.x == 0) {
        prefix = 0;
        nSel = 0;
        need = want;
    }
    __syncthreads();
    if (want > 0) {
        for (int shift = 56; shift >= 0; shift -= 8) {
            for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
            __syncthreads();
            const unsigned long long hiMask = shift == 56 ? 0ull : (~0ull << (shift + 8));
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                const unsigned long long key = keys[i];
                if (key != ~0ull && (key & hiMask) == prefix) atomicAdd(&hist[(key >> shift) & 0xFFu], 1u);
            }
            __syncthreads();
            if (threadIdx.x < 32) {
                // d = the first digit below 255 whose inclusive count reaches `need`, else 255;
                // c = the count of the digits before d.  Lane l holds digits 8l .. 8l + 7.
                const uint32_t lane = threadIdx.x;
                uint32_t h[8], incl[8], run = 0;
#pragma unroll
                for (uint32_t j = 0; j < 8; j++) {
                    h[j] = hist[8 * lane + j];
                    run += h[j];
                    incl[j] = run;
                }
                uint32_t before = run;
#pragma unroll
                for (uint32_t off = 1; off < 32; off <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, before, off);
                    if (lane >= off) before += v;
                }
                before -= run; // digits of the lower lanes
                const uint32_t nd = need;
                uint32_t jHit = 8, cHit = 0;
#pragma unroll
                for (int j = 7; j >= 0; j--) {
                    if (8 * lane + j < 255 && before + incl[j] >= nd) {
                        jHit = j;
                        cHit = before + incl[j] - h[j];
                    }
                }
                const uint32_t hitLanes = __ballot_sync(0xFFFFFFFFu, jHit < 8);
                const uint32_t src = hitLanes ? __ffs(hitLanes) - 1 : 31u;
                if (lane == src) {
                    const uint32_t d = hitLanes ? 8 * lane + jHit : 255u;
                    const uint32_t c = hitLanes ? cHit : before + incl[6]; // else digits 0 .. 254
                    need = nd - c;
                    prefix |= static_cast<unsigned long long>(d) << shift;
                }
            }
            __syncthreads();
        }
        // prefix is the want-th smallest key; keys are distinct, so exactly `want` are <= prefix
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned long long key = keys[i];
            if (key <= prefix) {
                const uint32_t s = atomicAdd(&nSel, 1u);
                if (s < selCap) sel[s] = key;
            }
        }
    }
    __syncthreads();
    const uint32_t m = nSel < selCap ? nSel : selCap;
    uint32_t mPow2 = 1;
    while (mPow2 < m) mPow2 <<= 1;
    for (uint32_t i = m + threadIdx.x; i < mPow2; i += blockDim.x) sel[i] = ~0ull;
    __syncthreads();
    bitonicSortShared(sel, mPow2);
}

__device__ __forceinline__ void writeResults(const ScoreParams& P, uint32_t q, const unsigned long long* sel, uint32_t want)
{
    for (uint32_t i = threadIdx.x; i < want; i += blockDim.x) {
        P.outDocs[uint64_t(q) * P.k + i] = static_cast<uint32_t>(sel[i]);
        P.outScores[uint64_t(q) * P.k + i] = fromOrderedBits(static_cast<uint32_t>(sel[i] >> 32));
    }
    if (threadIdx.x == 0) P.outCount[q] = want;
}

// One CTA per (query, range of shardDocs documents).  The accumulators of the range live in
// shared memory (9 B per document).  Grouped segments hand the CTA the leaf postings of its
// csrPerCta shards only (one range per leaf word); upper-level words read their group's range
// and keep the CTA's documents.  A single-layout segment is walked by every CTA of the query,
// each keeping the postings of its range.  kSharded = false: one range holds every document and
// no posting needs the range test.
template <bool kSharded, uint32_t kThreads>
__global__ void __launch_bounds__(kThreads, kThreads >= 1024 ? 1 : 1024 / kThreads) scoreKernel(ScoreParams P)
{
    extern __shared__ unsigned long long dyn[];
    __shared__ uint32_t nTouched;
    __shared__ uint32_t nextBatch; // entry batches are handed to warps as they finish
    __shared__ unsigned long long sel[kMaxK];
    const uint32_t q = P.order ? P.order[blockIdx.x] : blockIdx.x;
    const uint32_t shard = blockIdx.y;
    const uint32_t docBeg = kSharded ? shard * P.shardDocs : 0u;
    const uint32_t nLocal = kSharded ? min(P.shardDocs, P.nDocs - docBeg) : P.nDocs;
    // Accumulators through a generic pointer: the 64-bit atomics on it measured faster than
    // the shared-window form the compiler picks for a known shared-memory address.
    unsigned long long* acc;
    asm("mov.b64 %0, %1;" : "=l"(acc) : "l"(reinterpret_cast<unsigned long long*>(dyn)));
    for (uint32_t i = threadIdx.x; i < nLocal; i += blockDim.x) acc[i] = 0;
    if (threadIdx.x == 0) {
        nTouched = 0;
        nextBatch = 0;
    }
    __syncthreads();

    const uint32_t lane = threadIdx.x & 31u;
    const Entry* ent = P.entries + (P.qOff[q] - P.qOff[0]) * P.L;
    const uint32_t ne = P.entryCount[q];
    const float qRcp = P.qRcpF[q];
    // The CTA's pair range of a word (leaves [lo, hi)) in segment s.
    const uint32_t groupOf = docBeg / kSmemDocs, shardInGroup = (docBeg % kSmemDocs) / kShardDocs;
    auto wordRange = [&](int s, uint64_t lo, uint64_t hi, bool leafLevel, uint32_t& a, uint32_t& b) {
        const SegmentView& v = P.seg[s];
        if (!v.grouped) {
            a = v.leafOff[lo];
            b = v.leafOff[hi];
            return;
        }
        const uint32_t g = groupOf - v.groupBeg;
        if (g >= v.nGroups) {
            a = b = 0;
            return;
        }
        const uint32_t* t = v.leafOff + uint64_t(g) * P.nbLeaves * kGroupShards;
        if (leafLevel) {
            a = t[lo * kGroupShards + shardInGroup];
            b = t[lo * kGroupShards + shardInGroup + P.csrPerCta];
        } else {
            a = t[lo * kGroupShards];
            b = t[hi * kGroupShards];
        }
    };
    auto addPair = [&](uint64_t pr, float qv) {
        const uint32_t i = static_cast<uint32_t>(pr >> 32) - docBeg;
        if (!kSharded || i < nLocal) addTerm(acc, i, termOf(qv, __uint_as_float(static_cast<uint32_t>(pr))));
    };
    // A leaf word's list [a, b) by the whole warp, eight pairs per lane in flight.
    auto leafList = [&](const uint64_t* pairs, uint32_t a, uint32_t b, float qv) {
        uint32_t p = a + lane;
        for (; p + 224 < b; p += 256) {
            uint64_t pr[8];
#pragma unroll
            for (int u = 0; u < 8; u++) pr[u] = pairs[p + 32 * u];
#pragma unroll
            for (int u = 0; u < 8; u++) addPair(pr[u], qv);
        }
        for (; p < b; p += 32) addPair(pairs[p], qv);
    };
    // Virtual inverted file of a non-leaf word: the union of the leaf lists below it, counted
    // per document (DataBase.cpp:150-164).  A document lives in one segment only, and the skip
    // rule keeps the union short, so each lane scans the range for the documents of this shard
    // whose first pair it holds.
    auto virtualList = [&](int s, uint32_t a, uint32_t b, float w, float qv) {
        const uint64_t* pairs = P.seg[s].pairs;
        for (uint32_t p = a + lane; p < b; p += 32) {
            const uint32_t slot = static_cast<uint32_t>(pairs[p] >> 32);
            if (kSharded && slot - docBeg >= nLocal) continue;
            bool first = true;
            for (uint32_t r = a; r < p && first; r++) first = static_cast<uint32_t>(pairs[r] >> 32) != slot;
            if (!first) continue;
            uint32_t tf = 0;
            for (uint32_t r = p; r < b; r++)
                if (static_cast<uint32_t>(pairs[r] >> 32) == slot) tf += P.seg[s].tf[r];
            const float d = float(tf) * w * P.rcpF[slot];
            addTerm(acc, slot - docBeg, termOf(qv, d));
        }
    };
    // Entries in batches of 32 per warp: lane j fetches entry base + j, its weight and its
    // offsets in both segments, so these loads overlap instead of chaining entry after entry.
    // Leaf lists shorter than kFlatList are then walked as one range over the batch (lane t of
    // a round takes pair t of the concatenated lists, kFlatDepth pairs per lane in flight);
    // longer lists and non-leaf words go one at a time with the whole warp.
    for (;;) {
        uint32_t batch = 0;
        if (lane == 0) batch = atomicAdd(&nextBatch, 1u);
        const uint32_t base = __shfl_sync(0xFFFFFFFFu, batch, 0) * 32u;
        if (base >= ne) break;
        const uint32_t e = base + lane;
        const bool valid = e < ne;
        float qv = 0.f, w = 0.f;
        bool leaf = false;
        uint32_t a0 = 0, b0 = 0, a1 = 0, b1 = 0;
        if (valid) {
            const Entry en = ent[e];
            w = P.weights[en.widx];
            qv = float(en.run) * w * qRcp;
            leaf = en.level == P.L - 1;
            const uint64_t span = ipowDev(P.B, P.L - 1 - en.level);
            const uint64_t lo = uint64_t(en.word) * span;
            wordRange(0, lo, lo + span, leaf, a0, b0);
            wordRange(1, lo, lo + span, leaf, a1, b1);
        }
        const uint32_t len = (b0 - a0) + (b1 - a1);
        const bool flat = valid && leaf && len < kFlatList;
        for (uint32_t one = __ballot_sync(0xFFFFFFFFu, valid && !flat); one != 0; one &= one - 1) {
            const uint32_t j = __ffs(one) - 1;
            const uint32_t ja0 = __shfl_sync(0xFFFFFFFFu, a0, j), jb0 = __shfl_sync(0xFFFFFFFFu, b0, j);
            const uint32_t ja1 = __shfl_sync(0xFFFFFFFFu, a1, j), jb1 = __shfl_sync(0xFFFFFFFFu, b1, j);
            const float jq = __shfl_sync(0xFFFFFFFFu, qv, j), jw = __shfl_sync(0xFFFFFFFFu, w, j);
            if (__shfl_sync(0xFFFFFFFFu, leaf, j)) {
                leafList(P.seg[0].pairs, ja0, jb0, jq);
                leafList(P.seg[1].pairs, ja1, jb1, jq);
            } else {
                virtualList(0, ja0, jb0, jw, jq);
                virtualList(1, ja1, jb1, jw, jq);
            }
        }
        const uint32_t c0 = flat ? b0 - a0 : 0u;
        const uint32_t cnt = flat ? len : 0u;
        uint32_t incl = cnt;
#pragma unroll
        for (uint32_t off = 1; off < 32; off <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
            if (lane >= off) incl += v;
        }
        const uint32_t excl = incl - cnt;
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        for (uint32_t f0 = 0; f0 < total; f0 += 32u * kFlatDepth) {
            uint64_t pr[kFlatDepth];
            float pq[kFlatDepth];
#pragma unroll
            for (uint32_t u = 0; u < kFlatDepth; u++) {
                const uint32_t t = f0 + 32u * u + lane;
                // owner lane: the last j with excl_j <= t (excl is non-decreasing; it holds pairs)
                uint32_t j = 0;
#pragma unroll
                for (uint32_t step = 16; step > 0; step >>= 1) {
                    const uint32_t v = __shfl_sync(0xFFFFFFFFu, excl, j + step);
                    if (v <= t) j += step;
                }
                const uint32_t off = t - __shfl_sync(0xFFFFFFFFu, excl, j);
                const uint32_t jc0 = __shfl_sync(0xFFFFFFFFu, c0, j);
                const uint32_t ja0 = __shfl_sync(0xFFFFFFFFu, a0, j), ja1 = __shfl_sync(0xFFFFFFFFu, a1, j);
                pq[u] = __shfl_sync(0xFFFFFFFFu, qv, j);
                pr[u] = 0;
                if (t < total) pr[u] = off < jc0 ? P.seg[0].pairs[ja0 + off] : P.seg[1].pairs[ja1 + off - jc0];
            }
#pragma unroll
            for (uint32_t u = 0; u < kFlatDepth; u++)
                if (f0 + 32u * u + lane < total) addPair(pr[u], pq[u]);
        }
    }
    __syncthreads();

    // Keys: ordered score bits << 32 | document id.  Ties in score go to the lower document id;
    // untouched documents get ~0.
    uint32_t myTouched = 0;
    for (uint32_t i = threadIdx.x; i < nLocal; i += blockDim.x) {
        unsigned long long key = ~0ull;
        if (acc[i] != 0) { // touched: every term adds at least one unit
            const double sum = static_cast<double>(static_cast<long long>(acc[i])) / kFixScale;
            const float score = float(sum + 2.0f);
            key = (static_cast<unsigned long long>(orderedBits(score)) << 32) | P.slotDoc[docBeg + i];
            myTouched++;
        }
        acc[i] = key;
    }
    atomicAdd(&nTouched, myTouched);
    __syncthreads();
    const uint32_t want = P.k < nTouched ? P.k : nTouched;
    unsigned long long* selp = P.selGlobal ? P.selGlobal + (uint64_t(q) * gridDim.y + shard) * P.selStride : sel;
    selectSmallest(acc, nLocal, want, selp, P.selGlobal ? P.selStride : kMaxK);
    if (P.cand == nullptr) {
        writeResults(P, q, selp, want);
    } else {
        unsigned long long* c = P.cand + (uint64_t(q) * gridDim.y + shard) * P.k;
        for (uint32_t i = threadIdx.x; i < P.k; i += blockDim.x) c[i] = i < want ? selp[i] : ~0ull;
    }
}

// The k best of the shards' candidates of each query (one CTA per query).
__global__ void __launch_bounds__(kScoreThreads) mergeKernel(ScoreParams P, uint32_t shards)
{
    __shared__ uint32_t nValid;
    __shared__ unsigned long long sel[kMaxK];
    const uint32_t q = blockIdx.x;
    const unsigned long long* c = P.cand + uint64_t(q) * shards * P.k;
    const uint32_t n = shards * P.k;
    if (threadIdx.x == 0) nValid = 0;
    __syncthreads();
    uint32_t mine = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) mine += c[i] != ~0ull ? 1u : 0u;
    atomicAdd(&nValid, mine);
    __syncthreads();
    const uint32_t want = P.k < nValid ? P.k : nValid;
    unsigned long long* selp = P.selGlobal ? P.selGlobal + uint64_t(q) * shards * P.selStride : sel;
    selectSmallest(c, n, want, selp, P.selGlobal ? P.selStride : kMaxK);
    writeResults(P, q, selp, want);
}

// Device memory from the library's stream-ordered pool, grown on a stream (keeping a prefix).
class PoolBuffer
{
public:
    PoolBuffer() = default;
    PoolBuffer(const PoolBuffer&) = delete;
    PoolBuffer& operator=(const PoolBuffer&) = delete;
    template <typename T>
    T* as() const { return static_cast<T*>(mPtr); }
    void* get() const { return mPtr; }
    // Ensures capacity >= need bytes; the first `keep` bytes survive a reallocation.
    void reserve(size_t need, size_t keep, cudaStream_t s)
    {
        if (need <= mCap) return;
        const size_t cap = std::max(need, mCap + mCap / 2);
        void* p = nullptr;
        RBW_CUDA(cudaMallocFromPoolAsync(&p, cap, libraryPool(), s));
        if (keep && mPtr) RBW_CUDA(cudaMemcpyAsync(p, mPtr, keep, cudaMemcpyDeviceToDevice, s));
        if (mPtr) RBW_CUDA(cudaFreeAsync(mPtr, s));
        mPtr = p;
        mCap = cap;
    }
    void release(cudaStream_t s)
    {
        if (mPtr) cudaFreeAsync(mPtr, s);
        mPtr = nullptr;
        mCap = 0;
    }

private:
    void* mPtr = nullptr;
    size_t mCap = 0;
};

struct Segment {
    PoolBuffer leafOff;   // u32 offset table (segIndex) + 1 tail entry
    PoolBuffer pairs;     // u64 slot << 32 | float bits of the leaf-level document entry
    PoolBuffer tf;        // u32 per pair
    uint32_t slotBeg = 0, slotEnd = 0;
    bool grouped = false; // grouped layout: groups of kSmemDocs documents, leaves, shards
    uint32_t groupBeg = 0, nGroups = 1;
    SegmentView view() const
    {
        return SegmentView{leafOff.as<uint32_t>(), pairs.as<uint64_t>(), tf.as<uint32_t>(), grouped ? 1u : 0u,
                           groupBeg, nGroups};
    }
};

// The kernels' dynamic shared-memory limits are raised once per device to the largest size any
// launch uses: changing a function's attribute between launches can wait for that function's
// launches in flight on other streams.
constexpr int kPrepSmemMax = int(kMaxDocDesc) * 4;
constexpr int kScoreSmemMax = int(kSmemDocs) * 8;

template <uint32_t kThreads>
void launchScore(bool sharded, dim3 grid, size_t smem, cudaStream_t stream, const ScoreParams& P)
{
    static std::atomic<uint64_t> setS{0}, setU{0};
    if (sharded) {
        setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(scoreKernel<true, kThreads>), kScoreSmemMax, setS);
        scoreKernel<true, kThreads><<<grid, kThreads, smem, stream>>>(P);
    } else {
        setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(scoreKernel<false, kThreads>), kScoreSmemMax,
                                       setU);
        scoreKernel<false, kThreads><<<grid, kThreads, smem, stream>>>(P);
    }
    RBW_CUDA(cudaGetLastError());
}

} // namespace

// ------------------------------------------------------------------ host class
class DataBase
{
public:
    explicit DataBase(const Vocabulary& v) : mB{v.branch()}, mL{v.levels()}
    {
        mNbLeaves = ipowDev(mB, mL);
        mNbWords = levelBeg(mB, mL) * mB;
        if (mNbLeaves >= 0xFFFFFFFFull) throw Error(kUnsupported, "tree too large for a DataBase");
        mWeights.reset(mNbWords * 4);
        RBW_CUDA(cudaMemcpy(mWeights.get(), v.weights().data(), mNbWords * 4, cudaMemcpyHostToDevice));
        mHostDocOff.push_back(0);
        RBW_CUDA(cudaStreamCreateWithFlags(&mStream, cudaStreamNonBlocking));
        RBW_CUDA(cudaEventCreateWithFlags(&mIndexReady, cudaEventDisableTiming));
        // empty index: zero offsets in both segments, zero word counts
        for (Segment* sg : {&mMain, &mDelta}) {
            sg->leafOff.reserve((mNbLeaves + 1) * 4, 0, mStream);
            sg->pairs.reserve(8, 0, mStream);
            sg->tf.reserve(4, 0, mStream);
            RBW_CUDA(cudaMemsetAsync(sg->leafOff.get(), 0, (mNbLeaves + 1) * 4, mStream));
        }
        mMainLeafPost.reserve(mNbLeaves * 8, 0, mStream);
        RBW_CUDA(cudaMemsetAsync(mMainLeafPost.get(), 0, mNbLeaves * 8, mStream));
        mWordPost.reserve(mNbWords * 8, 0, mStream);
        RBW_CUDA(cudaMemsetAsync(mWordPost.get(), 0, mNbWords * 8, mStream));
        for (PoolBuffer* b : {&mDocOff, &mDocPairs, &mPairCount, &mRcpF, &mSlotDoc}) b->reserve(64, 0, mStream);
        RBW_CUDA(cudaMemsetAsync(mDocOff.get(), 0, 8, mStream));
        RBW_CUDA(cudaEventRecord(mIndexReady, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
    }
    ~DataBase()
    {
        waitQueriesOnStream();
        for (PoolBuffer* b : {&mDocOff, &mDocPairs, &mPairCount, &mRcpF, &mSlotDoc, &mMainLeafPost, &mWordPost,
                              &mMain.leafOff, &mMain.pairs, &mMain.tf, &mDelta.leafOff, &mDelta.pairs, &mDelta.tf})
            b->release(mStream);
        cudaStreamSynchronize(mStream);
        for (auto& kv : mQueryEvents) cudaEventDestroy(kv.second);
        cudaEventDestroy(mIndexReady);
        cudaStreamDestroy(mStream);
    }

    void addDoc(uint32_t id, const uint32_t* leaves, uint32_t n)
    {
        std::unique_lock<std::shared_mutex> lk(mMu);
        checkDoc(id, leaves, n);
        stageLocked(id, leaves, n);
    }
    void addDocs(const uint32_t* ids, const uint32_t* leaves, const uint64_t* off, uint32_t nDocs)
    {
        std::unique_lock<std::shared_mutex> lk(mMu);
        // validate the whole batch first: a failed call adds nothing
        std::unordered_map<uint32_t, uint32_t> seen;
        for (uint32_t d = 0; d < nDocs; d++) {
            if (off[d + 1] < off[d] || off[d + 1] - off[d] > 0xFFFFFFFFull)
                throw Error(kInvalidArg, "bad document offsets");
            checkDoc(ids[d], leaves + off[d], static_cast<uint32_t>(off[d + 1] - off[d]));
            if (!seen.emplace(ids[d], d).second) throw Error(kDuplicate, "Duplicate document index");
        }
        for (uint32_t d = 0; d < nDocs; d++)
            stageLocked(ids[d], leaves + off[d], static_cast<uint32_t>(off[d + 1] - off[d]));
    }

    // Host leaves in, host results out (the reference's query).  Synchronous.
    uint32_t query(const uint32_t* leaves, uint32_t n, uint32_t k, uint32_t* docs, float* scores)
    {
        for (uint32_t i = 0; i < n; i++)
            if (leaves[i] >= mNbLeaves) throw Error(kInvalidArg, "leaf index out of range");
        if (k == 0) return 0;
        const uint64_t off[2] = {0, n};
        cudaStream_t s = mStream;
        void* din = nullptr;
        void* dout = nullptr;
        RBW_CUDA(cudaMallocFromPoolAsync(&din, 16 + size_t(n) * 4, libraryPool(), s));
        RBW_CUDA(cudaMallocFromPoolAsync(&dout, size_t(k) * 8 + 16, libraryPool(), s));
        uint32_t got = 0;
        try {
            uint64_t* dOff = static_cast<uint64_t*>(din);
            uint32_t* dLeaves = reinterpret_cast<uint32_t*>(dOff + 2);
            RBW_CUDA(cudaMemcpyAsync(dOff, off, 16, cudaMemcpyHostToDevice, s));
            if (n) RBW_CUDA(cudaMemcpyAsync(dLeaves, leaves, size_t(n) * 4, cudaMemcpyHostToDevice, s));
            uint32_t* dDocs = static_cast<uint32_t*>(dout);
            float* dScores = reinterpret_cast<float*>(dDocs + k);
            uint32_t* dCount = reinterpret_cast<uint32_t*>(dScores + k);
            queryBatched(dLeaves, dOff, 1, k, dDocs, dScores, dCount, s, off);
            RBW_CUDA(cudaMemcpyAsync(&got, dCount, 4, cudaMemcpyDeviceToHost, s));
            RBW_CUDA(cudaStreamSynchronize(s));
            if (got) {
                RBW_CUDA(cudaMemcpyAsync(docs, dDocs, size_t(got) * 4, cudaMemcpyDeviceToHost, s));
                if (scores) RBW_CUDA(cudaMemcpyAsync(scores, dScores, size_t(got) * 4, cudaMemcpyDeviceToHost, s));
            }
        } catch (...) {
            cudaFreeAsync(din, s);
            cudaFreeAsync(dout, s);
            cudaStreamSynchronize(s);
            throw;
        }
        RBW_CUDA(cudaFreeAsync(din, s));
        RBW_CUDA(cudaFreeAsync(dout, s));
        RBW_CUDA(cudaStreamSynchronize(s));
        return got;
    }

    // Device leaves and offsets in, device results out; the kernels run asynchronously on
    // `stream`.  hostOff, if given, is a host copy of dOff (saves reading the offsets back).
    void queryBatched(const uint32_t* dLeaves, const uint64_t* dOff, uint32_t nq, uint32_t k, uint32_t* dDocs,
                      float* dScores, uint32_t* dCount, cudaStream_t stream, const uint64_t* hostOff = nullptr)
    {
        if (nq == 0) return;
        if (dOff == nullptr || dCount == nullptr || (k && (dDocs == nullptr || dScores == nullptr)))
            throw Error(kInvalidArg, "null argument");
        std::vector<uint64_t> off;
        if (hostOff == nullptr) {
            off.resize(size_t(nq) + 1);
            RBW_CUDA(cudaMemcpyAsync(off.data(), dOff, off.size() * 8, cudaMemcpyDeviceToHost, stream));
            RBW_CUDA(cudaStreamSynchronize(stream));
            hostOff = off.data();
        }
        uint32_t maxN = 0, maxBig = 0;
        std::vector<uint32_t> bigQ; // queries sorted in global memory
        for (uint32_t q = 0; q < nq; q++) {
            if (hostOff[q + 1] < hostOff[q] || hostOff[q + 1] - hostOff[q] > 0xFFFFFFFFull)
                throw Error(kInvalidArg, "bad query offsets");
            const uint32_t m = static_cast<uint32_t>(hostOff[q + 1] - hostOff[q]);
            if (m > kMaxDocDesc) {
                bigQ.push_back(q);
                maxBig = std::max(maxBig, m);
            } else {
                maxN = std::max(maxN, m);
            }
        }
        if ((maxN || maxBig) && dLeaves == nullptr) throw Error(kInvalidArg, "null argument");
        const uint64_t totalLeaves = hostOff[nq] - hostOff[0];
        updateIndex();
        std::shared_lock<std::shared_mutex> lk(mMu);
        RBW_CUDA(cudaStreamWaitEvent(stream, mIndexReady, 0));
        if (k == 0) {
            RBW_CUDA(cudaMemsetAsync(dCount, 0, size_t(nq) * 4, stream));
            return;
        }
        const uint32_t nDocs = mIndexed;
        cudaMemPool_t pool = libraryPool();
        int dev = 0, sms = 0;
        RBW_CUDA(cudaGetDevice(&dev));
        RBW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        // Document range per scoring CTA.  With grouped inverted files it is csrPerCta shards of
        // kShardDocs documents: the most (up to a group of kSmemDocs documents) that still gives
        // one CTA per SM, so a small batch spreads over the GPU; with one inverted file per
        // segment, kSmemDocs documents (every CTA of a query walks the whole list).
        uint32_t csrPerCta = 1, shardDocs = std::min(std::max(nDocs, 1u), kSmemDocs);
        if (groupedIndex()) {
            csrPerCta = kSmemDocs / kShardDocs;
            while (csrPerCta > 1 &&
                   uint64_t(nq) * ((nDocs + csrPerCta * kShardDocs - 1) / (csrPerCta * kShardDocs)) < uint64_t(sms))
                csrPerCta /= 2;
            shardDocs = std::min(std::max(nDocs, 1u), csrPerCta * kShardDocs);
        }
        const uint32_t shards = std::max(1u, (nDocs + shardDocs - 1) / shardDocs);
        const size_t entBytes = std::max<uint64_t>(totalLeaves, 1) * mL * sizeof(Entry);
        const size_t candBytes = shards > 1 ? size_t(nq) * shards * k * 8 : 16;
        const uint32_t selStride = k > kMaxK ? nextPow2(k) : 0u;
        const size_t selBytes = k > kMaxK ? size_t(nq) * shards * selStride * 8 : 16;
        const uint32_t bigStride = maxBig ? nextPow2(maxBig) : 0u;
        const size_t bigBytes = bigQ.empty() ? 16 : bigQ.size() * (size_t(bigStride) + 1) * 4;
        void *ent = nullptr, *cnt = nullptr, *qr = nullptr, *cand = nullptr, *selG = nullptr, *big = nullptr;
        void* wk = nullptr;
        RBW_CUDA(cudaMallocFromPoolAsync(&wk, size_t(nq) * 12, pool, stream));
        unsigned long long* work = static_cast<unsigned long long*>(wk);
        uint32_t* order = reinterpret_cast<uint32_t*>(work + nq);
        RBW_CUDA(cudaMallocFromPoolAsync(&ent, entBytes, pool, stream));
        RBW_CUDA(cudaMallocFromPoolAsync(&cnt, size_t(nq) * 4, pool, stream));
        RBW_CUDA(cudaMallocFromPoolAsync(&qr, size_t(nq) * 4, pool, stream));
        RBW_CUDA(cudaMallocFromPoolAsync(&cand, candBytes, pool, stream));
        RBW_CUDA(cudaMallocFromPoolAsync(&selG, selBytes, pool, stream));
        RBW_CUDA(cudaMallocFromPoolAsync(&big, bigBytes, pool, stream));
        {
            ScopedKernelTimer timer(kTimedScore, stream);
            std::optional<ScopedKernelTimer> prepTimer(std::in_place, kTimedScorePrep, stream);
            const size_t prepSmem = size_t(nextPow2(std::max(maxN, 1u))) * 4;
            static std::atomic<uint64_t> setPrep{0};
            setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(queryPrepKernel), kPrepSmemMax, setPrep);
            queryPrepKernel<<<nq, kPrepThreads, prepSmem, stream>>>(
                dLeaves, dOff, nullptr, nullptr, 0u, mWeights.as<float>(), skipCounts(), mB, mL,
                mNbLeaves, k, static_cast<float*>(qr), static_cast<Entry*>(ent), static_cast<uint32_t*>(cnt), work);
            RBW_CUDA(cudaGetLastError());
            if (!bigQ.empty()) {
                // queries above kMaxDocDesc descriptors: one CTA each, sorted in global memory
                uint32_t* qList = static_cast<uint32_t*>(big);
                uint32_t* gkeys = qList + bigQ.size();
                RBW_CUDA(cudaMemcpyAsync(qList, bigQ.data(), bigQ.size() * 4, cudaMemcpyHostToDevice, stream));
                queryPrepKernel<<<static_cast<uint32_t>(bigQ.size()), kPrepThreads, 0, stream>>>(
                    dLeaves, dOff, qList, gkeys, bigStride, mWeights.as<float>(), skipCounts(),
                    mB, mL, mNbLeaves, k, static_cast<float*>(qr), static_cast<Entry*>(ent),
                    static_cast<uint32_t*>(cnt), work);
                RBW_CUDA(cudaGetLastError());
            }
            prepTimer.reset();
            ScoreParams P{};
            P.entries = static_cast<const Entry*>(ent);
            P.entryCount = static_cast<const uint32_t*>(cnt);
            P.qOff = dOff;
            P.qRcpF = static_cast<const float*>(qr);
            P.weights = mWeights.as<float>();
            P.seg[0] = mMain.view();
            P.seg[1] = mDelta.view();
            P.csrPerCta = csrPerCta;
            P.nbLeaves = mNbLeaves;
            P.rcpF = mRcpF.as<float>();
            P.slotDoc = mSlotDoc.as<uint32_t>();
            P.nDocs = nDocs;
            P.shardDocs = shardDocs;
            P.B = mB;
            P.L = mL;
            P.k = k;
            P.cand = shards > 1 ? static_cast<unsigned long long*>(cand) : nullptr;
            P.selGlobal = k > kMaxK ? static_cast<unsigned long long*>(selG) : nullptr;
            P.selStride = selStride;
            // more queries than one wave of scoring CTAs: start the longest ones first
            if (nq > uint32_t(sms) && nq <= kOrderMax) {
                workOrderKernel<<<1, 1024, 0, stream>>>(work, nq, order);
                RBW_CUDA(cudaGetLastError());
                P.order = order;
            }
            P.outDocs = dDocs;
            P.outScores = dScores;
            P.outCount = dCount;
            // 1,024 threads per CTA whatever its document range: the pair walk is bound by load
            // latency, so a query split over few CTAs needs every warp an SM can hold
            const size_t smem = size_t(shardDocs) * 8;
            launchScore<kScoreThreads>(shards > 1, dim3(nq, shards), smem, stream, P);
            if (shards > 1) {
                ScopedKernelTimer mergeTimer(kTimedScoreMerge, stream);
                mergeKernel<<<nq, kScoreThreads, 0, stream>>>(P, shards);
                RBW_CUDA(cudaGetLastError());
            }
        }
        RBW_CUDA(cudaFreeAsync(ent, stream));
        RBW_CUDA(cudaFreeAsync(cnt, stream));
        RBW_CUDA(cudaFreeAsync(qr, stream));
        RBW_CUDA(cudaFreeAsync(cand, stream));
        RBW_CUDA(cudaFreeAsync(selG, stream));
        RBW_CUDA(cudaFreeAsync(big, stream));
        RBW_CUDA(cudaFreeAsync(wk, stream));
        recordQuery(stream);
    }

    // Subtree posting counts of every word ([levelBeg(L)][B], leaf level included) of this
    // database, as its skip rule uses them.
    std::vector<uint64_t> wordPostings()
    {
        updateIndex();
        std::shared_lock<std::shared_mutex> lk(mMu);
        std::vector<uint64_t> out(mNbWords);
        RBW_CUDA(cudaMemcpyAsync(out.data(), mWordPost.get(), mNbWords * 8, cudaMemcpyDeviceToHost, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
        return out;
    }

    // Counts the skip rule uses instead of this database's own (nullptr: back to its own).  A
    // database holding one shard of a document set takes the counts summed over all shards, so
    // every shard skips exactly the words the whole set would (DataBase.cpp:125).
    void setWordPostings(const uint64_t* host)
    {
        std::unique_lock<std::shared_mutex> lk(mMu);
        if (host == nullptr) {
            mSkipExternal = false;
            return;
        }
        waitQueriesOnStream();
        if (mSkipCounts.get() == nullptr) mSkipCounts.reset(mNbWords * 8);
        RBW_CUDA(cudaMemcpyAsync(mSkipCounts.get(), host, mNbWords * 8, cudaMemcpyHostToDevice, mStream));
        RBW_CUDA(cudaEventRecord(mIndexReady, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
        mSkipExternal = true;
    }

    uint32_t nbDocs()
    {
        std::shared_lock<std::shared_mutex> lk(mMu);
        return static_cast<uint32_t>(mHostIds.size());
    }
    uint64_t nbPostings()
    {
        std::shared_lock<std::shared_mutex> lk(mMu);
        return mHostDocOff.back();
    }
    // Documents in the main and delta segments of the current index (diagnostics).
    void segments(uint32_t* mainDocs, uint32_t* deltaDocs)
    {
        updateIndex();
        std::shared_lock<std::shared_mutex> lk(mMu);
        if (mainDocs) *mainDocs = mMain.slotEnd - mMain.slotBeg;
        if (deltaDocs) *deltaDocs = mDelta.slotEnd - mDelta.slotBeg;
    }

    float docRcp(uint32_t id)
    {
        updateIndex();
        std::shared_lock<std::shared_mutex> lk(mMu);
        const auto it = mSlotOf.find(id);
        if (it == mSlotOf.end()) throw Error(kInvalidArg, "unknown document");
        float v = 0;
        RBW_CUDA(cudaMemcpyAsync(&v, mRcpF.as<float>() + it->second, 4, cudaMemcpyDeviceToHost, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
        return v;
    }

    // A leaf's posting list as the reference stores it: document ids ascending, each repeated
    // tf times (DataBase.cpp:44-53).
    std::vector<uint32_t> postings(uint32_t leaf)
    {
        if (leaf >= mNbLeaves) throw Error(kInvalidArg, "leaf out of range");
        updateIndex();
        std::shared_lock<std::shared_mutex> lk(mMu);
        std::vector<uint32_t> out;
        std::vector<std::pair<const Segment*, uint32_t>> groups; // (segment, group)
        for (const Segment* sg : {&mMain, &mDelta})
            for (uint32_t g = 0; g < sg->nGroups; g++) groups.emplace_back(sg, g);
        for (const auto& [sg, g] : groups) {
            // the leaf's pairs of the whole group: [index(leaf, shard 0), index(leaf + 1, shard 0))
            const uint32_t slot = (sg->groupBeg + g) * kSmemDocs;
            const uint64_t i0 = segIndex(slot, leaf, sg->groupBeg, mNbLeaves, sg->grouped);
            const uint64_t i1 = segIndex(slot, uint64_t(leaf) + 1, sg->groupBeg, mNbLeaves, sg->grouped);
            uint32_t ab[2] = {0, 0};
            RBW_CUDA(cudaMemcpyAsync(&ab[0], sg->leafOff.as<uint32_t>() + i0, 4, cudaMemcpyDeviceToHost, mStream));
            RBW_CUDA(cudaMemcpyAsync(&ab[1], sg->leafOff.as<uint32_t>() + i1, 4, cudaMemcpyDeviceToHost, mStream));
            RBW_CUDA(cudaStreamSynchronize(mStream));
            if (ab[1] < ab[0]) throw Error(kInternal, "inconsistent posting offsets");
            std::vector<uint64_t> pr(ab[1] - ab[0]);
            std::vector<uint32_t> tf(pr.size());
            if (!pr.empty()) {
                RBW_CUDA(cudaMemcpyAsync(pr.data(), sg->pairs.as<uint64_t>() + ab[0], pr.size() * 8,
                                         cudaMemcpyDeviceToHost, mStream));
                RBW_CUDA(cudaMemcpyAsync(tf.data(), sg->tf.as<uint32_t>() + ab[0], tf.size() * 4,
                                         cudaMemcpyDeviceToHost, mStream));
                RBW_CUDA(cudaStreamSynchronize(mStream));
            }
            for (size_t i = 0; i < pr.size(); i++) {
                if (tf[i] > mHostDocOff.back() || (pr[i] >> 32) >= mHostIds.size())
                    throw Error(kInternal, "inconsistent posting entry");
                out.insert(out.end(), tf[i], mHostIds[pr[i] >> 32]);
            }
        }
        std::sort(out.begin(), out.end());
        return out;
    }

private:
    void checkDoc(uint32_t id, const uint32_t* leaves, uint32_t n) const
    {
        if (mSlotOf.count(id)) throw Error(kDuplicate, "Duplicate document index"); // DataBase.cpp:41-43
        if (n && leaves == nullptr) throw Error(kInvalidArg, "null leaves");
        for (uint32_t i = 0; i < n; i++)
            if (leaves[i] >= mNbLeaves) throw Error(kInvalidArg, "leaf index out of range");
    }

    void stageLocked(uint32_t id, const uint32_t* leaves, uint32_t n)
    {
        mSlotOf.emplace(id, static_cast<uint32_t>(mHostIds.size()));
        mHostIds.push_back(id);
        mStage.insert(mStage.end(), leaves, leaves + n);
        mHostDocOff.push_back(mHostDocOff.back() + n);
        if (n <= kMaxDocDesc) mStageMaxN = std::max(mStageMaxN, n);
    }

    // Makes the stream wait for every query launched since the last index update.
    void waitQueriesOnStream()
    {
        std::lock_guard<std::mutex> lk(mEvMu);
        for (auto& kv : mQueryEvents) RBW_CUDA(cudaStreamWaitEvent(mStream, kv.second, 0));
    }

    void recordQuery(cudaStream_t stream)
    {
        std::lock_guard<std::mutex> lk(mEvMu);
        auto it = mQueryEvents.find(stream);
        if (it == mQueryEvents.end()) {
            cudaEvent_t ev = nullptr;
            RBW_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            it = mQueryEvents.emplace(stream, ev).first;
        }
        RBW_CUDA(cudaEventRecord(it->second, stream));
    }

    // How a segment's inverted file is laid out: grouped (segIndex; each scoring CTA then reads
    // only its shards' leaf postings), one CSR for the segment, or grouped while those tables
    // stay small next to the postings themselves.
    enum class SegLayout { kAuto, kGrouped, kSingle };

    // CSR of the documents [s0, s1) into `sg`; their per-leaf posting counts into leafPost.
    void buildSegment(Segment& sg, uint32_t s0, uint32_t s1, unsigned long long* leafPost, SegLayout layout)
    {
        const uint64_t pairsUpper = mHostDocOff[s1] - mHostDocOff[s0];
        if (pairsUpper >= 0xFFFFFFFFull) throw Error(kUnsupported, "more than 2^32 postings in one segment");
        sg.slotBeg = s0;
        sg.slotEnd = s1;
        sg.grouped = false;
        sg.groupBeg = 0;
        sg.nGroups = 1;
        if (s1 > s0 && layout != SegLayout::kSingle) {
            const uint32_t first = s0 / kSmemDocs, last = (s1 - 1) / kSmemDocs;
            const uint64_t tableBytes = (uint64_t(last - first + 1) * mNbLeaves * kGroupShards + 1) * 4;
            const bool small = tableBytes <= std::max<uint64_t>(kShardTableMinBytes, pairsUpper * 12);
            const bool allowed = tunedValue(kTuneDbShardTables, mB, mL, s1 - s0) == 1;
            if (layout == SegLayout::kGrouped || (allowed && small)) {
                sg.grouped = true;
                sg.groupBeg = first;
                sg.nGroups = last - first + 1;
            }
        }
        const uint64_t entries = sg.grouped ? uint64_t(sg.nGroups) * mNbLeaves * kGroupShards : mNbLeaves;
        sg.leafOff.reserve((entries + 1) * 4, 0, mStream);
        sg.pairs.reserve(std::max<uint64_t>(pairsUpper, 1) * 8, 0, mStream);
        sg.tf.reserve(std::max<uint64_t>(pairsUpper, 1) * 4, 0, mStream);
        void* tmp = nullptr;
        const size_t cntBytes = entries * 4;
        const size_t scanBytes = scanTempWords(entries) * 4;
        RBW_CUDA(cudaMallocFromPoolAsync(&tmp, 2 * cntBytes + scanBytes, libraryPool(), mStream));
        uint32_t* leafPairCnt = static_cast<uint32_t*>(tmp);
        uint32_t* cursor = leafPairCnt + entries;
        uint32_t* scanTmp = cursor + entries;
        RBW_CUDA(cudaMemsetAsync(leafPairCnt, 0, 2 * cntBytes, mStream));
        RBW_CUDA(cudaMemsetAsync(leafPost, 0, mNbLeaves * 8, mStream));
        if (s1 > s0) {
            segCountKernel<<<s1 - s0, kSegThreads, 0, mStream>>>(mDocOff.as<uint64_t>(), mDocPairs.as<uint64_t>(),
                                                                mPairCount.as<uint32_t>(), s0, sg.groupBeg,
                                                                mNbLeaves, sg.grouped, leafPairCnt, leafPost);
            RBW_CUDA(cudaGetLastError());
        }
        uint32_t* leafOff = sg.leafOff.as<uint32_t>();
        exclusiveScanU32(leafPairCnt, leafOff, entries, scanTmp, mStream);
        leafOffTail<<<1, 1, 0, mStream>>>(leafPairCnt, leafOff, entries);
        if (s1 > s0) {
            segScatterKernel<<<s1 - s0, kSegThreads, 0, mStream>>>(
                mDocOff.as<uint64_t>(), mDocPairs.as<uint64_t>(), mPairCount.as<uint32_t>(), s0, sg.groupBeg,
                mNbLeaves, sg.grouped, mWeights.as<float>() + levelBeg(mB, mL - 1) * mB, mRcpF.as<float>(), leafOff,
                cursor,
                sg.pairs.as<uint64_t>(), sg.tf.as<uint32_t>());
        }
        RBW_CUDA(cudaGetLastError());
        RBW_CUDA(cudaFreeAsync(tmp, mStream));
    }

    // Brings the device index up to date with the staged documents.  Enqueues work on the
    // database stream only; queries order themselves after it through mIndexReady.
    void updateIndex()
    {
        {
            std::shared_lock<std::shared_mutex> lk(mMu);
            if (mIndexed == mHostIds.size()) return;
        }
        std::unique_lock<std::shared_mutex> lk(mMu);
        const uint32_t s0 = mIndexed;
        const uint32_t s1 = static_cast<uint32_t>(mHostIds.size());
        if (s0 == s1) return;
        ScopedKernelTimer timer(kTimedIndex, mStream);
        waitQueriesOnStream();
        const uint64_t p0 = mHostDocOff[s0], p1 = mHostDocOff[s1];
        // 1. per-document arrays, grown in place
        mDocOff.reserve((uint64_t(s1) + 1) * 8, (uint64_t(s0) + 1) * 8, mStream);
        mDocPairs.reserve(std::max<uint64_t>(p1, 1) * 8, p0 * 8, mStream);
        mPairCount.reserve(uint64_t(s1) * 4, uint64_t(s0) * 4, mStream);
        mRcpF.reserve(uint64_t(s1) * 4, uint64_t(s0) * 4, mStream);
        mSlotDoc.reserve(uint64_t(s1) * 4, uint64_t(s0) * 4, mStream);
        RBW_CUDA(cudaMemcpyAsync(mDocOff.as<uint64_t>() + s0 + 1, mHostDocOff.data() + s0 + 1,
                                 uint64_t(s1 - s0) * 8, cudaMemcpyHostToDevice, mStream));
        RBW_CUDA(cudaMemcpyAsync(mSlotDoc.as<uint32_t>() + s0, mHostIds.data() + s0, uint64_t(s1 - s0) * 4,
                                 cudaMemcpyHostToDevice, mStream));
        void* newLeaves = nullptr;
        RBW_CUDA(cudaMallocFromPoolAsync(&newLeaves, std::max<uint64_t>(p1 - p0, 1) * 4, libraryPool(), mStream));
        if (p1 > p0)
            RBW_CUDA(cudaMemcpyAsync(newLeaves, mStage.data(), (p1 - p0) * 4, cudaMemcpyHostToDevice, mStream));
        const size_t smem = size_t(nextPow2(std::max(mStageMaxN, 1u))) * 4;
        static std::atomic<uint64_t> setDoc{0};
        setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(docPrepKernel), kPrepSmemMax, setDoc);
        docPrepKernel<<<s1 - s0, kPrepThreads, smem, mStream>>>(
            static_cast<const uint32_t*>(newLeaves), mDocOff.as<uint64_t>(), s0, nullptr, nullptr, 0u,
            mWeights.as<float>(), mB, mL, mNbLeaves, mRcpF.as<float>(), mDocPairs.as<uint64_t>(),
            mPairCount.as<uint32_t>());
        RBW_CUDA(cudaGetLastError());
        // documents above kMaxDocDesc descriptors: one CTA each, sorted in global memory
        std::vector<uint32_t> bigSlots;
        uint64_t maxBig = 0;
        for (uint32_t s = s0; s < s1; s++) {
            const uint64_t m = mHostDocOff[s + 1] - mHostDocOff[s];
            if (m > kMaxDocDesc) {
                bigSlots.push_back(s);
                maxBig = std::max(maxBig, m);
            }
        }
        if (!bigSlots.empty()) {
            const uint32_t stride = nextPow2(static_cast<uint32_t>(maxBig));
            void* big = nullptr;
            RBW_CUDA(cudaMallocFromPoolAsync(&big, bigSlots.size() * (size_t(stride) + 1) * 4, libraryPool(), mStream));
            uint32_t* slotList = static_cast<uint32_t*>(big);
            RBW_CUDA(cudaMemcpyAsync(slotList, bigSlots.data(), bigSlots.size() * 4, cudaMemcpyHostToDevice, mStream));
            docPrepKernel<<<static_cast<uint32_t>(bigSlots.size()), kPrepThreads, 0, mStream>>>(
                static_cast<const uint32_t*>(newLeaves), mDocOff.as<uint64_t>(), s0, slotList,
                slotList + bigSlots.size(), stride, mWeights.as<float>(), mB, mL, mNbLeaves, mRcpF.as<float>(),
                mDocPairs.as<uint64_t>(), mPairCount.as<uint32_t>());
            RBW_CUDA(cudaGetLastError());
            RBW_CUDA(cudaFreeAsync(big, mStream));
        }
        RBW_CUDA(cudaFreeAsync(newLeaves, mStream));
        mStage.clear();
        mStageMaxN = 0;

        // 2. segments: compact everything into main when the delta outgrows its share
        unsigned long long* leafWords = mWordPost.as<unsigned long long>() + levelBeg(mB, mL - 1) * mB;
        const uint32_t mainEnd = mMain.slotEnd;
        if (s1 - mainEnd > std::max(kDeltaMinDocs, mainEnd / kDeltaFraction)) {
            buildSegment(mMain, 0, s1, mMainLeafPost.as<unsigned long long>(), SegLayout::kAuto);
            buildSegment(mDelta, s1, s1, leafWords, SegLayout::kAuto);
            RBW_CUDA(cudaMemcpyAsync(leafWords, mMainLeafPost.get(), mNbLeaves * 8, cudaMemcpyDeviceToDevice,
                                     mStream));
        } else {
            void* deltaPost = nullptr;
            RBW_CUDA(cudaMallocFromPoolAsync(&deltaPost, mNbLeaves * 8, libraryPool(), mStream));
            // the delta follows the main segment's layout, so a scoring CTA sees one kind
            const SegLayout layout = mainEnd == 0 ? SegLayout::kAuto
                                     : mMain.grouped ? SegLayout::kGrouped : SegLayout::kSingle;
            buildSegment(mDelta, mainEnd, s1, static_cast<unsigned long long*>(deltaPost), layout);
            leafPostCombine<<<blocks(mNbLeaves, 256), 256, 0, mStream>>>(
                mMainLeafPost.as<unsigned long long>(), static_cast<unsigned long long*>(deltaPost), leafWords,
                mNbLeaves);
            RBW_CUDA(cudaFreeAsync(deltaPost, mStream));
        }
        // 3. subtree posting counts of the upper levels
        for (uint32_t level = mL - 1; level-- > 0;) {
            wordPostKernel<<<blocks(ipowDev(mB, level + 1), 256), 256, 0, mStream>>>(
                mWordPost.as<unsigned long long>(), mB, level);
        }
        RBW_CUDA(cudaGetLastError());
        RBW_CUDA(cudaEventRecord(mIndexReady, mStream));
        mIndexed = s1;
    }

    // Every segment holding documents has the grouped layout (none holds any: false).
    bool groupedIndex() const
    {
        const bool mainDocs = mMain.slotEnd > mMain.slotBeg, deltaDocs = mDelta.slotEnd > mDelta.slotBeg;
        return (mainDocs || deltaDocs) && (!mainDocs || mMain.grouped) && (!deltaDocs || mDelta.grouped);
    }

    const unsigned long long* skipCounts() const
    {
        return mSkipExternal ? mSkipCounts.as<unsigned long long>() : mWordPost.as<unsigned long long>();
    }

    uint32_t mB, mL;
    uint64_t mNbLeaves = 0, mNbWords = 0;
    DeviceBuffer mWeights;
    DeviceBuffer mSkipCounts;      // counts set by setWordPostings
    bool mSkipExternal = false;
    // host state
    std::vector<uint32_t> mHostIds;        // slot -> document id
    std::vector<uint64_t> mHostDocOff;     // slot -> first posting (prefix sums of sizes)
    std::unordered_map<uint32_t, uint32_t> mSlotOf;
    std::vector<uint32_t> mStage;          // leaves of documents [mIndexed, nSlots)
    uint32_t mStageMaxN = 0;
    uint32_t mIndexed = 0;                 // documents in the device index
    // device state (library pool, ordered on mStream)
    PoolBuffer mDocOff, mDocPairs, mPairCount, mRcpF, mSlotDoc;
    Segment mMain, mDelta;
    PoolBuffer mMainLeafPost, mWordPost;
    cudaStream_t mStream = nullptr;
    cudaEvent_t mIndexReady = nullptr;
    std::unordered_map<cudaStream_t, cudaEvent_t> mQueryEvents;
    std::mutex mEvMu;
    std::shared_mutex mMu;
};

} // namespace rbw

struct rbw_database {
    std::unique_ptr<rbw::DataBase> db;
};

namespace {
rbw::DataBase& dbOf(const rbw_database* h)
{
    if (h == nullptr || !h->db) throw rbw::Error(rbw::kInvalidArg, "null database handle");
    return *h->db;
}
} // namespace

extern "C" {

int rbw_db_create(const rbw_vocabulary* voc, rbw_database** out)
{
    return rbw::runGuarded([&] {
        if (out == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output handle");
        *out = nullptr;
        *out = new rbw_database{std::make_unique<rbw::DataBase>(rbw::vocabularyOf(voc))};
    });
}

void rbw_db_destroy(rbw_database* db) { delete db; }

int rbw_db_add(rbw_database* db, uint32_t idx_doc, const uint32_t* host_leaves, uint32_t n)
{
    return rbw::runGuarded([&] { dbOf(db).addDoc(idx_doc, host_leaves, n); });
}

int rbw_db_add_batch(rbw_database* db, const uint32_t* doc_ids, const uint32_t* host_leaves, const uint64_t* offsets,
                     uint32_t n_docs)
{
    return rbw::runGuarded([&] {
        if (n_docs && (doc_ids == nullptr || offsets == nullptr)) throw rbw::Error(rbw::kInvalidArg, "null argument");
        dbOf(db).addDocs(doc_ids, host_leaves, offsets, n_docs);
    });
}

int rbw_db_query(const rbw_database* db, const uint32_t* host_leaves, uint32_t n, uint32_t max_results,
                 uint32_t* out_docs, float* out_scores, uint32_t* n_out)
{
    return rbw::runGuarded([&] {
        if ((host_leaves == nullptr && n) || (out_docs == nullptr && max_results) || n_out == nullptr)
            throw rbw::Error(rbw::kInvalidArg, "null argument");
        *n_out = dbOf(db).query(host_leaves, n, max_results, out_docs, out_scores);
    });
}

int rbw_db_query_and_add(rbw_database* db, uint32_t idx_doc, const uint32_t* host_leaves, uint32_t n,
                         uint32_t max_results, uint32_t* out_docs, float* out_scores, uint32_t* n_out)
{
    return rbw::runGuarded([&] {
        if ((host_leaves == nullptr && n) || (out_docs == nullptr && max_results) || n_out == nullptr)
            throw rbw::Error(rbw::kInvalidArg, "null argument");
        auto& d = dbOf(db);
        *n_out = d.query(host_leaves, n, max_results, out_docs, out_scores); // DataBase.cpp:192-197
        d.addDoc(idx_doc, host_leaves, n);
    });
}

int rbw_db_query_batched(const rbw_database* db, const uint32_t* dev_leaves, const uint64_t* dev_offsets,
                         uint32_t n_queries, uint32_t max_results, uint32_t* dev_docs, float* dev_scores,
                         uint32_t* dev_counts, void* stream)
{
    return rbw::runGuarded([&] {
        dbOf(db).queryBatched(dev_leaves, dev_offsets, n_queries, max_results, dev_docs, dev_scores, dev_counts,
                              static_cast<cudaStream_t>(stream));
    });
}

int rbw_db_query_batched_host_offsets(const rbw_database* db, const uint32_t* dev_leaves, const uint64_t* dev_offsets,
                                      const uint64_t* host_offsets, uint32_t n_queries, uint32_t max_results,
                                      uint32_t* dev_docs, float* dev_scores, uint32_t* dev_counts, void* stream)
{
    return rbw::runGuarded([&] {
        if (host_offsets == nullptr) throw rbw::Error(rbw::kInvalidArg, "null host offsets");
        dbOf(db).queryBatched(dev_leaves, dev_offsets, n_queries, max_results, dev_docs, dev_scores, dev_counts,
                              static_cast<cudaStream_t>(stream), host_offsets);
    });
}

int rbw_db_info(const rbw_database* db, uint32_t* n_docs, uint64_t* n_postings)
{
    return rbw::runGuarded([&] {
        auto& d = dbOf(db);
        if (n_docs) *n_docs = d.nbDocs();
        if (n_postings) *n_postings = d.nbPostings();
    });
}

int rbw_db_segments(const rbw_database* db, uint32_t* main_docs, uint32_t* delta_docs)
{
    return rbw::runGuarded([&] { dbOf(db).segments(main_docs, delta_docs); });
}

int rbw_db_doc_rcp(const rbw_database* db, uint32_t idx_doc, float* rcp)
{
    return rbw::runGuarded([&] {
        if (rcp == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        *rcp = dbOf(db).docRcp(idx_doc);
    });
}

int rbw_db_word_postings(const rbw_database* db, uint64_t* host_counts)
{
    return rbw::runGuarded([&] {
        if (host_counts == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        const auto v = dbOf(db).wordPostings();
        std::memcpy(host_counts, v.data(), v.size() * 8);
    });
}

int rbw_db_set_word_postings(rbw_database* db, const uint64_t* host_counts)
{
    return rbw::runGuarded([&] { dbOf(db).setWordPostings(host_counts); });
}

int rbw_db_postings(const rbw_database* db, uint32_t leaf, uint32_t* out, uint32_t capacity, uint32_t* n)
{
    return rbw::runGuarded([&] {
        const auto p = dbOf(db).postings(leaf);
        if (n) *n = static_cast<uint32_t>(p.size());
        if (out) std::memcpy(out, p.data(), std::min<size_t>(capacity, p.size()) * 4);
    });
}

} // extern "C"
