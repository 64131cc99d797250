// Device-resident inverted file and hierarchical tf-idf scoring (reference: DataBase.cpp:39-197).
//
// Index (rebuilt on the device when documents were added since the last query):
//   * docPrepKernel, one CTA per document: sorts its leaf words in shared memory, computes the
//     L1 norm of its weight vector over all levels in the reference's order (levels leaf->root,
//     descriptors in ascending leaf order, double sum; DataBase.cpp:54-68) and run-length
//     encodes (leaf, tf);
//   * (slot, tf) pairs are scattered into per-leaf CSR segments.  The pairs of a leaf are the
//     reference's sorted posting list with repeated document ids folded into tf;
//   * subtree posting counts of every word (with multiplicity) feed the reference's level skip
//     rule: a non-leaf word is scored only if its subtree holds < 16 + 4k postings
//     (DataBase.h:60-61, DataBase.cpp:125).
// Queries (any number per launch, uneven sizes):
//   * queryPrepKernel, one CTA per query: sort, query L1 norm (same order as documents), and
//     the (level, word, run) entries that survive the skip rule;
//   * scoreKernel, one CTA per query: warps take entries and add, for every document in the
//     entry's postings, the reference's term |q - d| - (q + d), q = run*w*qRcp and
//     d = tf*w*dRcp in float (DataBase.cpp:117,127-131).  Each document's terms are summed in
//     64-bit fixed point (2^-56 units), so the sum does not depend on the order in which warps
//     add them; the score is float(sum + 2) (DataBase.cpp:170-174); the k best are chosen by a
//     radix select on (score, document id).
#include "capi_internal.h"
#include "kmeans.cuh"
#include "timing.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <shared_mutex>
#include <unordered_map>
#include <vector>

namespace rbw {
namespace {

constexpr uint32_t kMaxDocDesc = 32768;   // descriptors per document or query (in-CTA sort)
constexpr uint32_t kPrepThreads = 512;
constexpr uint32_t kScoreThreads = 512;
constexpr uint32_t kSmemDocs = 20480;     // per-document accumulators kept in shared memory
constexpr uint32_t kMaxK = 1024;
constexpr double kFixScale = 72057594037927936.0; // 2^56
constexpr size_t kGlobalAccBudget = size_t(1) << 30; // accumulators of one scoring launch

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

// Ascending bitonic sort of nPow2 keys in shared memory (all threads of the CTA take part).
template <typename T>
__device__ void bitonicSortShared(T* keys, uint32_t nPow2)
{
    for (uint32_t k = 2; k <= nPow2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < nPow2; i += blockDim.x) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const T a = keys[i], b = keys[ixj];
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
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

// Double sum of the weights of every (level, descriptor) in the reference's order.
__device__ double l1NormSequential(const uint32_t* sorted, uint32_t n, const float* weights, uint32_t B, uint32_t L)
{
    double norm = 0;
    uint64_t span = 1;
    for (uint32_t it = 0; it < L; it++) {
        const uint32_t level = L - 1 - it;
        const float* lw = weights + levelBegDev(B, level) * B;
        for (uint32_t i = 0; i < n; i++) norm += lw[sorted[i] / span];
        span *= B;
    }
    return norm;
}

// ------------------------------------------------------------------ index build
__global__ void __launch_bounds__(kPrepThreads) docPrepKernel(const uint32_t* leaves, const uint64_t* off,
                                                              const float* weights, uint32_t B, uint32_t L,
                                                              uint64_t nbLeaves, float* rcpF, uint64_t* pairTmp,
                                                              uint32_t* pairCount, uint32_t* leafPairCnt,
                                                              unsigned long long* leafPostCnt)
{
    extern __shared__ uint32_t keys[];
    __shared__ uint32_t cnt, nValid;
    const uint32_t doc = blockIdx.x;
    const uint64_t beg = off[doc];
    if (threadIdx.x == 0) cnt = 0;
    const uint32_t n = loadAndSort(leaves + beg, static_cast<uint32_t>(off[doc + 1] - beg), keys, nbLeaves, &nValid);
    if (threadIdx.x == 0) rcpF[doc] = float(1 / l1NormSequential(keys, n, weights, B, L)); // DataBase.cpp:68
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t k = keys[i];
        if (i == 0 || keys[i - 1] != k) {
            uint32_t run = 1;
            while (i + run < n && keys[i + run] == k) run++;
            const uint32_t p = atomicAdd(&cnt, 1u);
            pairTmp[beg + p] = (uint64_t(k) << 32) | run;
            atomicAdd(&leafPairCnt[k], 1u);
            atomicAdd(&leafPostCnt[k], static_cast<unsigned long long>(run));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) pairCount[doc] = cnt;
}

__global__ void scatterPairsKernel(const uint64_t* off, const uint64_t* pairTmp, const uint32_t* pairCount,
                                   const uint32_t* leafOff, uint32_t* cursor, uint64_t* pairs)
{
    const uint32_t doc = blockIdx.x;
    const uint64_t beg = off[doc];
    for (uint32_t p = threadIdx.x; p < pairCount[doc]; p += blockDim.x) {
        const uint64_t v = pairTmp[beg + p];
        const uint32_t leaf = static_cast<uint32_t>(v >> 32);
        const uint32_t tf = static_cast<uint32_t>(v);
        const uint32_t pos = leafOff[leaf] + atomicAdd(&cursor[leaf], 1u);
        pairs[pos] = (uint64_t(doc) << 32) | tf;
    }
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

__global__ void leafOffTail(const uint32_t* leafPairCnt, uint32_t* leafOff, uint64_t nLeaves)
{
    leafOff[nLeaves] = leafOff[nLeaves - 1] + leafPairCnt[nLeaves - 1];
}

// ------------------------------------------------------------------ queries
__global__ void __launch_bounds__(kPrepThreads) queryPrepKernel(const uint32_t* qLeaves, const uint64_t* qOff,
                                                                const float* weights,
                                                                const unsigned long long* wordPost, uint32_t B,
                                                                uint32_t L, uint64_t nbLeaves, uint32_t k,
                                                                float* qRcpF, Entry* entries, uint32_t* entryCount)
{
    extern __shared__ uint32_t keys[];
    __shared__ uint32_t cnt, nValid;
    const uint32_t q = blockIdx.x;
    const uint64_t beg = qOff[q];
    Entry* out = entries + (beg - qOff[0]) * L;
    if (threadIdx.x == 0) cnt = 0;
    const uint32_t n = loadAndSort(qLeaves + beg, static_cast<uint32_t>(qOff[q + 1] - beg), keys, nbLeaves, &nValid);
    if (threadIdx.x == 0) qRcpF[q] = float(1 / l1NormSequential(keys, n, weights, B, L)); // DataBase.cpp:77-94
    uint64_t span = 1;
    const uint64_t limit = 16ull + 4ull * k; // DataBase.h:60-61, DataBase.cpp:125
    for (uint32_t it = 0; it < L; it++) {
        const uint32_t level = L - 1 - it;
        const uint64_t base = levelBegDev(B, level) * B;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t word = static_cast<uint32_t>(keys[i] / span);
            if (i == 0 || keys[i - 1] / span != word) {
                uint32_t run = 1;
                while (i + run < n && keys[i + run] / span == word) run++;
                const uint64_t widx = base + word;
                if (it == 0 || wordPost[widx] < limit) {
                    const uint32_t p = atomicAdd(&cnt, 1u);
                    out[p] = Entry{level, word, run, static_cast<uint32_t>(widx)};
                }
            }
        }
        span *= B;
    }
    __syncthreads();
    if (threadIdx.x == 0) entryCount[q] = cnt;
}

struct ScoreParams {
    const Entry* entries;
    const uint32_t* entryCount;
    const uint64_t* qOff;
    const float* qRcpF;
    const float* weights;
    const uint32_t* leafOff;
    const uint64_t* pairs;
    const float* rcpF;
    const uint32_t* slotDoc;
    uint32_t nDocs;
    uint32_t B;
    uint32_t L;
    uint32_t k;
    uint32_t qBase;             // first query of this launch
    unsigned long long* gAcc;   // [launch queries][nDocs] when the accumulators do not fit shared memory
    uint32_t* gBits;            // [launch queries][(nDocs + 31) / 32]
    uint32_t* outDocs;          // [nq][k]
    float* outScores;           // [nq][k]
    uint32_t* outCount;         // [nq]
};

__device__ __forceinline__ float termOf(float q, float d) { return fabsf(q - d) - (q + d); }

__device__ __forceinline__ void addTerm(unsigned long long* acc, uint32_t* bits, uint32_t slot, float term)
{
    const long long fx = llrint(static_cast<double>(term) * kFixScale);
    atomicAdd(&acc[slot], static_cast<unsigned long long>(fx));
    atomicOr(&bits[slot >> 5], 1u << (slot & 31u));
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

__global__ void __launch_bounds__(kScoreThreads) scoreKernel(ScoreParams P)
{
    extern __shared__ unsigned long long dyn[];
    __shared__ uint32_t hist[256];
    __shared__ unsigned long long prefix;
    __shared__ uint32_t need, nSel, nTouched;
    __shared__ unsigned long long sel[kMaxK];
    const uint32_t local = blockIdx.x;
    const uint32_t q = P.qBase + local;
    const uint32_t nWords = (P.nDocs + 31) / 32;
    const bool inSmem = P.gAcc == nullptr;
    unsigned long long* acc = inSmem ? dyn : P.gAcc + uint64_t(local) * P.nDocs;
    uint32_t* bits = inSmem ? reinterpret_cast<uint32_t*>(dyn + P.nDocs) : P.gBits + uint64_t(local) * nWords;
    for (uint32_t i = threadIdx.x; i < P.nDocs; i += blockDim.x) acc[i] = 0;
    for (uint32_t i = threadIdx.x; i < nWords; i += blockDim.x) bits[i] = 0;
    if (threadIdx.x == 0) nTouched = 0;
    __syncthreads();

    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nWarpsCta = blockDim.x >> 5;
    const Entry* ent = P.entries + (P.qOff[q] - P.qOff[0]) * P.L;
    const uint32_t ne = P.entryCount[q];
    const float qRcp = P.qRcpF[q];
    for (uint32_t e = warp; e < ne; e += nWarpsCta) {
        const Entry en = ent[e];
        const float w = P.weights[en.widx];
        const float qv = float(en.run) * w * qRcp;
        if (en.level == P.L - 1) {
            const uint32_t a = P.leafOff[en.word], b = P.leafOff[en.word + 1];
            for (uint32_t p = a + lane; p < b; p += 32) {
                const uint64_t pr = P.pairs[p];
                const uint32_t slot = static_cast<uint32_t>(pr >> 32);
                const float d = float(static_cast<uint32_t>(pr)) * w * P.rcpF[slot];
                addTerm(acc, bits, slot, termOf(qv, d));
            }
        } else {
            // Virtual inverted file of a non-leaf word: the union of the leaf lists below it,
            // counted per document (DataBase.cpp:150-164).  The skip rule keeps it short, so
            // each lane scans it for the documents it owns.
            const uint64_t span = ipowDev(P.B, P.L - 1 - en.level);
            const uint32_t a = P.leafOff[uint64_t(en.word) * span], b = P.leafOff[(uint64_t(en.word) + 1) * span];
            for (uint32_t p = a + lane; p < b; p += 32) {
                const uint32_t slot = static_cast<uint32_t>(P.pairs[p] >> 32);
                bool first = true;
                for (uint32_t r = a; r < p && first; r++) first = static_cast<uint32_t>(P.pairs[r] >> 32) != slot;
                if (!first) continue;
                uint32_t tf = 0;
                for (uint32_t r = p; r < b; r++) {
                    const uint64_t v = P.pairs[r];
                    if (static_cast<uint32_t>(v >> 32) == slot) tf += static_cast<uint32_t>(v);
                }
                const float d = float(tf) * w * P.rcpF[slot];
                addTerm(acc, bits, slot, termOf(qv, d));
            }
        }
    }
    __syncthreads();

    // Keys: ordered score bits << 32 | document id.  Ties in score go to the lower document id;
    // untouched documents get ~0.
    uint32_t myTouched = 0;
    for (uint32_t i = threadIdx.x; i < P.nDocs; i += blockDim.x) {
        unsigned long long key = ~0ull;
        if (bits[i >> 5] & (1u << (i & 31u))) {
            const double sum = static_cast<double>(static_cast<long long>(acc[i])) / kFixScale;
            const float score = float(sum + 2.0f);
            key = (static_cast<unsigned long long>(orderedBits(score)) << 32) | P.slotDoc[i];
            myTouched++;
        }
        acc[i] = key;
    }
    atomicAdd(&nTouched, myTouched);
    if (threadIdx.x == 0) {
        prefix = 0;
        nSel = 0;
    }
    __syncthreads();
    const uint32_t want = P.k < nTouched ? P.k : nTouched;
    if (threadIdx.x == 0) need = want;
    __syncthreads();
    if (want > 0) {
        // radix select of the want-th smallest key, 8 bits at a time
        for (int shift = 56; shift >= 0; shift -= 8) {
            for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
            __syncthreads();
            const unsigned long long hiMask = shift == 56 ? 0ull : (~0ull << (shift + 8));
            for (uint32_t i = threadIdx.x; i < P.nDocs; i += blockDim.x) {
                const unsigned long long key = acc[i];
                if (key != ~0ull && (key & hiMask) == prefix) atomicAdd(&hist[(key >> shift) & 0xFFu], 1u);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t c = 0, d = 0;
                for (; d < 255; d++) {
                    if (c + hist[d] >= need) break;
                    c += hist[d];
                }
                need -= c;
                prefix |= static_cast<unsigned long long>(d) << shift;
            }
            __syncthreads();
        }
        // prefix is the want-th smallest key; keys are distinct, so exactly `want` are <= prefix
        for (uint32_t i = threadIdx.x; i < P.nDocs; i += blockDim.x) {
            const unsigned long long key = acc[i];
            if (key <= prefix) {
                const uint32_t s = atomicAdd(&nSel, 1u);
                if (s < kMaxK) sel[s] = key;
            }
        }
    }
    __syncthreads();
    const uint32_t m = nSel < kMaxK ? nSel : kMaxK;
    uint32_t mPow2 = 1;
    while (mPow2 < m) mPow2 <<= 1;
    for (uint32_t i = m + threadIdx.x; i < mPow2; i += blockDim.x) sel[i] = ~0ull;
    __syncthreads();
    bitonicSortShared(sel, mPow2);
    for (uint32_t i = threadIdx.x; i < want; i += blockDim.x) {
        P.outDocs[uint64_t(q) * P.k + i] = static_cast<uint32_t>(sel[i]);
        P.outScores[uint64_t(q) * P.k + i] = fromOrderedBits(static_cast<uint32_t>(sel[i] >> 32));
    }
    if (threadIdx.x == 0) P.outCount[q] = want;
}

uint32_t blocks(uint64_t n, uint32_t t) { return static_cast<uint32_t>((n + t - 1) / t); }

} // namespace

// ------------------------------------------------------------------ host class
class DataBase
{
public:
    explicit DataBase(const Vocabulary& v) : mVoc{v}, mB{v.branch()}, mL{v.levels()}
    {
        mNbLeaves = ipowDev(mB, mL);
        mNbWords = levelBeg(mB, mL) * mB;
        mWeights.reset(mNbWords * 4);
        RBW_CUDA(cudaMemcpy(mWeights.get(), v.weights().data(), mNbWords * 4, cudaMemcpyHostToDevice));
        mHostOff.push_back(0);
        RBW_CUDA(cudaStreamCreateWithFlags(&mStream, cudaStreamNonBlocking));
    }
    ~DataBase()
    {
        if (mStream) cudaStreamDestroy(mStream);
    }

    void addDoc(uint32_t id, const uint32_t* leaves, uint32_t n)
    {
        std::unique_lock<std::shared_mutex> lk(mMu);
        checkDoc(id, leaves, n);
        appendLocked(id, leaves, n);
    }
    void addDocs(const uint32_t* ids, const uint32_t* leaves, const uint64_t* off, uint32_t nDocs)
    {
        std::unique_lock<std::shared_mutex> lk(mMu);
        // validate the whole batch first: a failed call adds nothing
        std::unordered_map<uint32_t, uint32_t> seen;
        for (uint32_t d = 0; d < nDocs; d++) {
            if (off[d + 1] < off[d] || off[d + 1] - off[d] > kMaxDocDesc)
                throw Error(kInvalidArg, "bad document offsets or document too large");
            checkDoc(ids[d], leaves + off[d], static_cast<uint32_t>(off[d + 1] - off[d]));
            if (!seen.emplace(ids[d], d).second) throw Error(kDuplicate, "Duplicate document index");
        }
        for (uint32_t d = 0; d < nDocs; d++)
            appendLocked(ids[d], leaves + off[d], static_cast<uint32_t>(off[d + 1] - off[d]));
    }

    // Host leaves in, host results out (the reference's query).  Synchronous.
    uint32_t query(const uint32_t* leaves, uint32_t n, uint32_t k, uint32_t* docs, float* scores)
    {
        if (n > kMaxDocDesc) throw Error(kUnsupported, "a query may hold at most 32768 descriptors");
        if (k > kMaxK) throw Error(kUnsupported, "maxNbResults above 1024 is not supported");
        for (uint32_t i = 0; i < n; i++)
            if (leaves[i] >= mNbLeaves) throw Error(kInvalidArg, "leaf index out of range");
        if (k == 0) return 0;
        const uint64_t off[2] = {0, n};
        cudaMemPool_t pool = libraryPool();
        const size_t inBytes = 16 + size_t(n) * 4;
        const size_t outBytes = size_t(k) * 8 + 16;
        void* din = nullptr;
        void* dout = nullptr;
        RBW_CUDA(cudaMallocFromPoolAsync(&din, inBytes, pool, mStream));
        RBW_CUDA(cudaMallocFromPoolAsync(&dout, outBytes, pool, mStream));
        uint32_t got = 0;
        try {
            uint64_t* dOff = static_cast<uint64_t*>(din);
            uint32_t* dLeaves = reinterpret_cast<uint32_t*>(dOff + 2);
            RBW_CUDA(cudaMemcpyAsync(dOff, off, 16, cudaMemcpyHostToDevice, mStream));
            if (n) RBW_CUDA(cudaMemcpyAsync(dLeaves, leaves, size_t(n) * 4, cudaMemcpyHostToDevice, mStream));
            uint32_t* dDocs = static_cast<uint32_t*>(dout);
            float* dScores = reinterpret_cast<float*>(dDocs + k);
            uint32_t* dCount = reinterpret_cast<uint32_t*>(dScores + k);
            queryBatched(dLeaves, dOff, 1, k, dDocs, dScores, dCount, mStream, off);
            RBW_CUDA(cudaMemcpyAsync(&got, dCount, 4, cudaMemcpyDeviceToHost, mStream));
            RBW_CUDA(cudaStreamSynchronize(mStream));
            if (got) {
                RBW_CUDA(cudaMemcpyAsync(docs, dDocs, size_t(got) * 4, cudaMemcpyDeviceToHost, mStream));
                if (scores)
                    RBW_CUDA(cudaMemcpyAsync(scores, dScores, size_t(got) * 4, cudaMemcpyDeviceToHost, mStream));
            }
        } catch (...) {
            cudaFreeAsync(din, mStream);
            cudaFreeAsync(dout, mStream);
            cudaStreamSynchronize(mStream);
            throw;
        }
        RBW_CUDA(cudaFreeAsync(din, mStream));
        RBW_CUDA(cudaFreeAsync(dout, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
        return got;
    }

    // Device leaves and offsets in, device results out; the kernels run asynchronously on
    // `stream`.  The index is first brought up to date (synchronously) if documents were added.
    // hostOff, if given, is a host copy of dOff (saves reading the offsets back).
    void queryBatched(const uint32_t* dLeaves, const uint64_t* dOff, uint32_t nq, uint32_t k, uint32_t* dDocs,
                      float* dScores, uint32_t* dCount, cudaStream_t stream, const uint64_t* hostOff = nullptr)
    {
        if (k > kMaxK) throw Error(kUnsupported, "maxNbResults above 1024 is not supported");
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
        uint32_t maxN = 0;
        for (uint32_t q = 0; q < nq; q++) {
            if (hostOff[q + 1] < hostOff[q] || hostOff[q + 1] - hostOff[q] > kMaxDocDesc)
                throw Error(kInvalidArg, "bad query offsets or query above 32768 descriptors");
            maxN = std::max<uint32_t>(maxN, static_cast<uint32_t>(hostOff[q + 1] - hostOff[q]));
        }
        if (maxN && dLeaves == nullptr) throw Error(kInvalidArg, "null argument");
        const uint64_t totalLeaves = hostOff[nq] - hostOff[0];
        ensureIndex();
        std::shared_lock<std::shared_mutex> lk(mMu);
        if (k == 0) {
            RBW_CUDA(cudaMemsetAsync(dCount, 0, size_t(nq) * 4, stream));
            return;
        }
        cudaMemPool_t pool = libraryPool();
        const uint32_t nWords = (mNbDocs + 31) / 32;
        const bool smemAcc = mNbDocs <= kSmemDocs;
        const size_t perQueryAcc = size_t(mNbDocs) * 8 + size_t(nWords) * 4;
        const uint32_t chunk =
            smemAcc ? nq : static_cast<uint32_t>(std::clamp<size_t>(kGlobalAccBudget / perQueryAcc, 1, nq));
        const size_t entBytes = std::max<uint64_t>(totalLeaves, 1) * mL * sizeof(Entry);
        const size_t accBytes = smemAcc ? 16 : size_t(chunk) * perQueryAcc + 16;
        void *ent = nullptr, *cnt = nullptr, *qr = nullptr, *acc = nullptr;
        RBW_CUDA(cudaMallocFromPoolAsync(&ent, entBytes, pool, stream));
        RBW_CUDA(cudaMallocFromPoolAsync(&cnt, size_t(nq) * 4, pool, stream));
        RBW_CUDA(cudaMallocFromPoolAsync(&qr, size_t(nq) * 4, pool, stream));
        RBW_CUDA(cudaMallocFromPoolAsync(&acc, accBytes, pool, stream));
        {
            ScopedKernelTimer timer(kTimedScore, stream);
            const size_t prepSmem = size_t(nextPow2(std::max(maxN, 1u))) * 4;
            RBW_CUDA(cudaFuncSetAttribute(queryPrepKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(prepSmem)));
            queryPrepKernel<<<nq, kPrepThreads, prepSmem, stream>>>(
                dLeaves, dOff, mWeights.as<float>(), mWordPost.as<unsigned long long>(), mB, mL, mNbLeaves, k,
                static_cast<float*>(qr), static_cast<Entry*>(ent), static_cast<uint32_t*>(cnt));
            RBW_CUDA(cudaGetLastError());
            ScoreParams P{};
            P.entries = static_cast<const Entry*>(ent);
            P.entryCount = static_cast<const uint32_t*>(cnt);
            P.qOff = dOff;
            P.qRcpF = static_cast<const float*>(qr);
            P.weights = mWeights.as<float>();
            P.leafOff = mLeafOff.as<uint32_t>();
            P.pairs = mPairs.as<uint64_t>();
            P.rcpF = mRcpF.as<float>();
            P.slotDoc = mSlotDoc.as<uint32_t>();
            P.nDocs = mNbDocs;
            P.B = mB;
            P.L = mL;
            P.k = k;
            P.outDocs = dDocs;
            P.outScores = dScores;
            P.outCount = dCount;
            size_t smem = 0;
            if (smemAcc) {
                smem = size_t(mNbDocs) * 8 + size_t(nWords) * 4;
            } else {
                P.gAcc = static_cast<unsigned long long*>(acc);
                P.gBits = reinterpret_cast<uint32_t*>(P.gAcc + size_t(chunk) * mNbDocs);
            }
            RBW_CUDA(cudaFuncSetAttribute(scoreKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            for (uint32_t q0 = 0; q0 < nq; q0 += chunk) {
                P.qBase = q0;
                scoreKernel<<<std::min(chunk, nq - q0), kScoreThreads, smem, stream>>>(P);
                RBW_CUDA(cudaGetLastError());
            }
        }
        RBW_CUDA(cudaFreeAsync(ent, stream));
        RBW_CUDA(cudaFreeAsync(cnt, stream));
        RBW_CUDA(cudaFreeAsync(qr, stream));
        RBW_CUDA(cudaFreeAsync(acc, stream));
    }

    uint32_t nbDocs()
    {
        std::shared_lock<std::shared_mutex> lk(mMu);
        return static_cast<uint32_t>(mHostIds.size());
    }
    uint64_t nbPostings()
    {
        std::shared_lock<std::shared_mutex> lk(mMu);
        return mHostLeaves.size();
    }

    float docRcp(uint32_t id)
    {
        ensureIndex();
        std::shared_lock<std::shared_mutex> lk(mMu);
        const auto it = mSlotOf.find(id);
        if (it == mSlotOf.end()) throw Error(kInvalidArg, "unknown document");
        float v = 0;
        RBW_CUDA(cudaMemcpy(&v, mRcpF.as<float>() + it->second, 4, cudaMemcpyDeviceToHost));
        return v;
    }

    // A leaf's posting list as the reference stores it: document ids ascending, each repeated
    // tf times (DataBase.cpp:44-53).
    std::vector<uint32_t> postings(uint32_t leaf)
    {
        if (leaf >= mNbLeaves) throw Error(kInvalidArg, "leaf out of range");
        ensureIndex();
        std::shared_lock<std::shared_mutex> lk(mMu);
        uint32_t ab[2] = {0, 0};
        RBW_CUDA(cudaMemcpy(ab, mLeafOff.as<uint32_t>() + leaf, 8, cudaMemcpyDeviceToHost));
        std::vector<uint64_t> pr(ab[1] - ab[0]);
        if (!pr.empty())
            RBW_CUDA(cudaMemcpy(pr.data(), mPairs.as<uint64_t>() + ab[0], pr.size() * 8, cudaMemcpyDeviceToHost));
        std::vector<uint32_t> out;
        for (const uint64_t v : pr) out.insert(out.end(), static_cast<uint32_t>(v), mHostIds[v >> 32]);
        std::sort(out.begin(), out.end());
        return out;
    }

private:
    void checkDoc(uint32_t id, const uint32_t* leaves, uint32_t n) const
    {
        if (mSlotOf.count(id)) throw Error(kDuplicate, "Duplicate document index"); // DataBase.cpp:41-43
        if (n > kMaxDocDesc) throw Error(kUnsupported, "a document may hold at most 32768 descriptors");
        if (n && leaves == nullptr) throw Error(kInvalidArg, "null leaves");
        for (uint32_t i = 0; i < n; i++)
            if (leaves[i] >= mNbLeaves) throw Error(kInvalidArg, "leaf index out of range");
    }

    void appendLocked(uint32_t id, const uint32_t* leaves, uint32_t n)
    {
        mSlotOf.emplace(id, static_cast<uint32_t>(mHostIds.size()));
        mHostIds.push_back(id);
        mHostLeaves.insert(mHostLeaves.end(), leaves, leaves + n);
        mHostOff.push_back(mHostLeaves.size());
        mMaxDocN = std::max(mMaxDocN, n);
        mDirty = true;
    }

    // Rebuilds the device index from all documents.  A rebuild replaces buffers that earlier
    // query launches may still read, so it first waits for the device to go idle.
    void ensureIndex()
    {
        {
            std::shared_lock<std::shared_mutex> lk(mMu);
            if (!mDirty) return;
        }
        std::unique_lock<std::shared_mutex> lk(mMu);
        if (!mDirty) return;
        if (mBuilt) RBW_CUDA(cudaDeviceSynchronize());
        const uint32_t nd = static_cast<uint32_t>(mHostIds.size());
        const uint64_t nl = mHostLeaves.size();
        if (nl > 0xFFFFFFFFull) throw Error(kUnsupported, "more than 2^32 postings");
        mNbDocs = nd;
        mSlotDoc.reset(std::max<uint64_t>(nd, 1) * 4);
        mRcpF.reset(std::max<uint64_t>(nd, 1) * 4);
        mLeafOff.reset((mNbLeaves + 1) * 4);
        mPairs.reset(std::max<uint64_t>(nl, 1) * 8);
        mWordPost.reset(mNbWords * 8);
        DeviceBuffer dLeaves(std::max<uint64_t>(nl, 1) * 4), dOff((uint64_t(nd) + 1) * 8);
        DeviceBuffer pairTmp(std::max<uint64_t>(nl, 1) * 8), pairCount(std::max<uint64_t>(nd, 1) * 4);
        DeviceBuffer leafPairCnt(mNbLeaves * 4), cursor(mNbLeaves * 4);
        DeviceBuffer scanTmp(scanTempWords(mNbLeaves) * 4);
        unsigned long long* leafPostCnt = mWordPost.as<unsigned long long>() + levelBeg(mB, mL - 1) * mB;
        {
            ScopedKernelTimer timer(kTimedIndex, mStream);
            if (nl)
                RBW_CUDA(cudaMemcpyAsync(dLeaves.get(), mHostLeaves.data(), nl * 4, cudaMemcpyHostToDevice, mStream));
            RBW_CUDA(cudaMemcpyAsync(dOff.get(), mHostOff.data(), (uint64_t(nd) + 1) * 8, cudaMemcpyHostToDevice,
                                     mStream));
            if (nd)
                RBW_CUDA(cudaMemcpyAsync(mSlotDoc.get(), mHostIds.data(), uint64_t(nd) * 4, cudaMemcpyHostToDevice,
                                         mStream));
            RBW_CUDA(cudaMemsetAsync(leafPairCnt.get(), 0, leafPairCnt.bytes(), mStream));
            RBW_CUDA(cudaMemsetAsync(mWordPost.get(), 0, mWordPost.bytes(), mStream));
            RBW_CUDA(cudaMemsetAsync(cursor.get(), 0, cursor.bytes(), mStream));
            if (nd) {
                const size_t smem = size_t(nextPow2(std::max(mMaxDocN, 1u))) * 4;
                RBW_CUDA(cudaFuncSetAttribute(docPrepKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
                docPrepKernel<<<nd, kPrepThreads, smem, mStream>>>(
                    dLeaves.as<uint32_t>(), dOff.as<uint64_t>(), mWeights.as<float>(), mB, mL, mNbLeaves,
                    mRcpF.as<float>(), pairTmp.as<uint64_t>(), pairCount.as<uint32_t>(), leafPairCnt.as<uint32_t>(),
                    leafPostCnt);
                RBW_CUDA(cudaGetLastError());
            }
            exclusiveScanU32(leafPairCnt.as<uint32_t>(), mLeafOff.as<uint32_t>(), mNbLeaves, scanTmp.as<uint32_t>(),
                             mStream);
            leafOffTail<<<1, 1, 0, mStream>>>(leafPairCnt.as<uint32_t>(), mLeafOff.as<uint32_t>(), mNbLeaves);
            if (nd) {
                scatterPairsKernel<<<nd, 256, 0, mStream>>>(dOff.as<uint64_t>(), pairTmp.as<uint64_t>(),
                                                            pairCount.as<uint32_t>(), mLeafOff.as<uint32_t>(),
                                                            cursor.as<uint32_t>(), mPairs.as<uint64_t>());
            }
            for (uint32_t level = mL - 1; level-- > 0;) {
                wordPostKernel<<<blocks(ipowDev(mB, level + 1), 256), 256, 0, mStream>>>(
                    mWordPost.as<unsigned long long>(), mB, level);
            }
            RBW_CUDA(cudaGetLastError());
        }
        RBW_CUDA(cudaStreamSynchronize(mStream));
        mDirty = false;
        mBuilt = true;
    }

    const Vocabulary& mVoc;
    uint32_t mB, mL;
    uint64_t mNbLeaves = 0, mNbWords = 0;
    DeviceBuffer mWeights, mWordPost;
    std::vector<uint32_t> mHostIds, mHostLeaves;
    std::vector<uint64_t> mHostOff;
    std::unordered_map<uint32_t, uint32_t> mSlotOf;
    uint32_t mMaxDocN = 0;
    bool mDirty = true;
    bool mBuilt = false;
    uint32_t mNbDocs = 0;
    DeviceBuffer mSlotDoc, mRcpF, mLeafOff, mPairs;
    cudaStream_t mStream = nullptr;
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

int rbw_db_info(const rbw_database* db, uint32_t* n_docs, uint64_t* n_postings)
{
    return rbw::runGuarded([&] {
        auto& d = dbOf(db);
        if (n_docs) *n_docs = d.nbDocs();
        if (n_postings) *n_postings = d.nbPostings();
    });
}

int rbw_db_doc_rcp(const rbw_database* db, uint32_t idx_doc, float* rcp)
{
    return rbw::runGuarded([&] {
        if (rcp == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        *rcp = dbOf(db).docRcp(idx_doc);
    });
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
