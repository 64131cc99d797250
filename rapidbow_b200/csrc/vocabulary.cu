// Vocabulary: tree storage, GPU hierarchical k-means build, lookup dispatch and the blob format.
//   build        : Vocabulary.cpp:32-121 + kmeans.cpp:27-225, all nodes of a level per launch
//   lookup       : Vocabulary.h:59-63 / Vocabulary.cpp:162-173
//   serialize    : Vocabulary.cpp:175-198 (byte-compatible for B = 16)
//   deserialize  : Vocabulary.cpp:126-157
#include "vocabulary.h"
#include "kmeans.cuh"
#include "tuning.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <thread>
#include <mutex>
#include <random>
#include <unordered_set>

namespace rbw {

DeviceBuffer::~DeviceBuffer()
{
    if (mPtr) cudaFree(mPtr);
}

void DeviceBuffer::reset(size_t bytes)
{
    if (mPtr) {
        cudaFree(mPtr);
        mPtr = nullptr;
        mBytes = 0;
    }
    if (bytes) {
        RBW_CUDA(cudaMalloc(&mPtr, bytes));
        mBytes = bytes;
    }
}

namespace {

constexpr uint32_t kBlobExtMagic = 0x32574252u;   // "RBW2": blobs with B != 16
constexpr uint32_t kBlobFloatMagic = 0x33574252u; // "RBW3": blobs with fp32 centers

__global__ void swizzleKernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, uint64_t nbNodes)
{
    // 128-byte swizzle of every 8-row atom: row r's 16-byte chunk c lands at chunk c ^ (r & 7),
    // the layout a TMA SWIZZLE_128B copy would write into 1024-byte-aligned shared memory.
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nbNodes * kMaxBranch * 8) return;
    const uint32_t chunk = i % 8;
    const uint64_t rowIdx = i / 8;
    const uint32_t row = rowIdx % kMaxBranch;
    const uint4 v = reinterpret_cast<const uint4*>(src)[i];
    reinterpret_cast<uint4*>(dst + rowIdx * kDims)[chunk ^ (row & 7u)] = v;
}

__global__ void normsKernel(const uint8_t* __restrict__ centers, int32_t* __restrict__ cnorm, uint64_t nbNodes,
                            uint32_t B)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nbNodes * kMaxBranch) return;
    if (i % kMaxBranch >= B) {
        cnorm[i] = kPadNorm;
        return;
    }
    const uint4* c = reinterpret_cast<const uint4*>(centers + i * kDims);
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint4 v = c[k];
        acc = __dp4a(v.x, v.x, acc);
        acc = __dp4a(v.y, v.y, acc);
        acc = __dp4a(v.z, v.z, acc);
        acc = __dp4a(v.w, v.w, acc);
    }
    cnorm[i] = static_cast<int32_t>(acc);
}

__global__ void padKernel(const uint8_t* __restrict__ canon, uint8_t* __restrict__ padded, uint64_t nbNodes, uint32_t B)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; // (node, slot, chunk)
    if (i >= nbNodes * kMaxBranch * 8) return;
    const uint32_t chunk = i % 8;
    const uint32_t b = (i / 8) % kMaxBranch;
    const uint64_t node = i / (8 * kMaxBranch);
    uint4 v = make_uint4(0, 0, 0, 0);
    if (b < B) v = reinterpret_cast<const uint4*>(canon + (node * B + b) * kDims)[chunk];
    reinterpret_cast<uint4*>(padded)[i] = v;
}

__global__ void padFloatKernel(const float* __restrict__ canon, float* __restrict__ padded, uint64_t nbNodes, uint32_t B)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; // (node, slot, dim)
    if (i >= nbNodes * kMaxBranch * kDims) return;
    const uint32_t d = i % kDims;
    const uint32_t b = (i / kDims) % kMaxBranch;
    const uint64_t node = i / (uint64_t(kDims) * kMaxBranch);
    padded[i] = b < B ? canon[(node * B + b) * kDims + d] : 0.f;
}

__global__ void roundCentersKernel(const float* __restrict__ f, uint8_t* __restrict__ u, uint64_t count, uint32_t B)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint32_t b = (i / kDims) % kMaxBranch;
    u[i] = b < B ? static_cast<uint8_t>(fminf(fmaxf(rintf(f[i]), 0.f), 255.f)) : uint8_t(0);
}

__global__ void iotaKernel(uint32_t* p, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) p[i] = static_cast<uint32_t>(i);
}

uint32_t blocksFor(uint64_t n, uint32_t t) { return static_cast<uint32_t>((n + t - 1) / t); }

} // namespace

// The reference's initial pick (kmeans.cpp:141-168): min(n, k) distinct members drawn from one
// default-seeded std::mt19937_64 that lives for the whole build (a fresh thread's
// thread_local engine), sorted and padded with the last pick.  The steps -- `rng() % n` into a
// hash set when n > 16*k, std::shuffle of 0..n-1 otherwise -- have to be the same calls on the
// same standard-library engine to reproduce the reference's trees.
uint32_t referencePick(std::mt19937_64& rng, uint32_t* dst, uint32_t space, uint32_t k)
{
    const uint32_t nbPick = std::min(space, k);
    if (nbPick * 16 < space) {
        std::unordered_set<uint32_t> picked;
        while (picked.size() != nbPick) picked.insert(static_cast<uint32_t>(rng() % space));
        std::copy_n(picked.begin(), nbPick, dst);
    } else {
        std::vector<uint32_t> all(space);
        std::iota(all.begin(), all.end(), 0u);
        std::shuffle(all.begin(), all.end(), rng);
        std::copy_n(all.begin(), nbPick, dst);
    }
    std::sort(dst, dst + nbPick);
    if (nbPick < k) std::fill(dst + nbPick, dst + k, nbPick != 0 ? dst[nbPick - 1] : 0u);
    return nbPick;
}

float idfWeight(uint32_t nbDoc, uint32_t occ)
{
    // Vocabulary.cpp:103-108
    return occ == 0 ? std::numeric_limits<float>::min()
                    : std::max(std::numeric_limits<float>::min(), std::log(float(nbDoc) / float(occ)));
}

void Vocabulary::allocate(uint32_t B, uint32_t L)
{
    if (B < 2 || B > kMaxBranch) throw Error(kUnsupported, "branch factor must be in [2, 16]");
    if (L < 1 || L > 8) throw Error(kUnsupported, "number of levels must be in [1, 8]");
    const uint64_t nodes = levelBeg(B, L);
    if (ipow(B, L) > 0xFFFFFFFFull) throw Error(kUnsupported, "leaf index does not fit 32 bits");
    mB = B;
    mL = L;
    mNbNodes = nodes;
    mCenters.reset(nodes * kMaxBranch * kDims);
    mCentersSw.reset(nodes * kMaxBranch * kDims);
    mCnorm.reset(nodes * kMaxBranch * sizeof(int32_t));
    mErrors.reset(sizeof(DeviceErrors));
    RBW_CUDA(cudaMemset(mErrors.get(), 0, sizeof(DeviceErrors)));
    mTree = DeviceTree{B, L, nodes, mCenters.as<uint8_t>(), mCentersSw.as<uint8_t>(), mCnorm.as<int32_t>()};
}

void Vocabulary::finalizeDevice(cudaStream_t stream)
{
    const uint64_t chunks = mNbNodes * kMaxBranch * 8;
    swizzleKernel<<<blocksFor(chunks, 256), 256, 0, stream>>>(mCenters.as<uint8_t>(), mCentersSw.as<uint8_t>(),
                                                              mNbNodes);
    normsKernel<<<blocksFor(mNbNodes * kMaxBranch, 256), 256, 0, stream>>>(mCenters.as<uint8_t>(),
                                                                           mCnorm.as<int32_t>(), mNbNodes, mB);
    RBW_CUDA(cudaGetLastError());
}

void Vocabulary::allocateFloat()
{
    const uint64_t nodes = mNbNodes;
    mCentersF.reset(nodes * kMaxBranch * kDims * sizeof(float));
    mSplit.reset(nodes * kSplitBytes);
    mCnF.reset(nodes * kMaxBranch * sizeof(float));
    mBound.reset(nodes * sizeof(float2));
    mRefined.reset(2 * sizeof(unsigned long long));
    RBW_CUDA(cudaMemset(mRefined.get(), 0, 2 * sizeof(unsigned long long)));
    mFloat = true;
}

void Vocabulary::roundFloatCenters(cudaStream_t stream)
{
    const uint64_t count = mNbNodes * kMaxBranch * kDims;
    roundCentersKernel<<<blocksFor(count, 256), 256, 0, stream>>>(mCentersF.as<float>(), mCenters.as<uint8_t>(), count,
                                                                  mB);
    RBW_CUDA(cudaGetLastError());
}

std::unique_ptr<Vocabulary> Vocabulary::fromHostF32(uint32_t B, uint32_t L, const float* centers,
                                                    const uint32_t* masks, const float* weights)
{
    std::unique_ptr<Vocabulary> v{new Vocabulary};
    v->allocate(B, L);
    v->allocateFloat();
    const uint64_t nodes = v->mNbNodes;
    DeviceBuffer canon(nodes * B * kDims * sizeof(float));
    RBW_CUDA(cudaMemcpy(canon.get(), centers, canon.bytes(), cudaMemcpyHostToDevice));
    padFloatKernel<<<blocksFor(nodes * kMaxBranch * kDims, 256), 256>>>(canon.as<float>(), v->mCentersF.as<float>(),
                                                                        nodes, B);
    RBW_CUDA(cudaGetLastError());
    launchPrepareFloatNodes(v->mCentersF.as<float>(), v->mSplit.as<uint8_t>(), v->mCnF.as<float>(),
                            v->mBound.as<float2>(), nodes, B, nullptr);
    v->roundFloatCenters(nullptr);
    v->mMasks.assign(masks, masks + nodes);
    v->mWeights.assign(weights, weights + nodes * B);
    v->finalizeDevice(nullptr);
    RBW_CUDA(cudaDeviceSynchronize());
    return v;
}

std::vector<float> Vocabulary::centersF32Host() const
{
    if (!mFloat) throw Error(kUnsupported, "the vocabulary has uint8 centers");
    std::vector<float> padded(mNbNodes * kMaxBranch * kDims);
    RBW_CUDA(cudaMemcpy(padded.data(), mCentersF.get(), padded.size() * sizeof(float), cudaMemcpyDeviceToHost));
    std::vector<float> out(mNbNodes * mB * kDims);
    for (uint64_t n = 0; n < mNbNodes; n++)
        std::memcpy(out.data() + n * mB * kDims, padded.data() + n * kMaxBranch * kDims,
                    size_t(mB) * kDims * sizeof(float));
    return out;
}

uint64_t Vocabulary::takeRefinedLookups() const
{
    if (!mFloat) return 0;
    unsigned long long v[2] = {0, 0};
    RBW_CUDA(cudaMemcpy(v, mRefined.get(), sizeof(v), cudaMemcpyDeviceToHost));
    RBW_CUDA(cudaMemset(mRefined.get(), 0, sizeof(v)));
    return v[0];
}

std::unique_ptr<Vocabulary> Vocabulary::fromHost(uint32_t B, uint32_t L, const uint8_t* centers, const uint32_t* masks,
                                                 const float* weights)
{
    std::unique_ptr<Vocabulary> v{new Vocabulary};
    v->allocate(B, L);
    const uint64_t nodes = v->mNbNodes;
    DeviceBuffer canon(nodes * B * kDims);
    RBW_CUDA(cudaMemcpy(canon.get(), centers, nodes * B * kDims, cudaMemcpyHostToDevice));
    padKernel<<<blocksFor(nodes * kMaxBranch * 8, 256), 256>>>(canon.as<uint8_t>(), v->mCenters.as<uint8_t>(), nodes, B);
    RBW_CUDA(cudaGetLastError());
    v->mMasks.assign(masks, masks + nodes);
    v->mWeights.assign(weights, weights + nodes * B);
    v->finalizeDevice(nullptr);
    RBW_CUDA(cudaDeviceSynchronize());
    return v;
}

std::vector<uint8_t> Vocabulary::centersHost() const
{
    std::vector<uint8_t> padded(mNbNodes * kMaxBranch * kDims);
    RBW_CUDA(cudaMemcpy(padded.data(), mCenters.get(), padded.size(), cudaMemcpyDeviceToHost));
    std::vector<uint8_t> out(mNbNodes * mB * kDims);
    for (uint64_t n = 0; n < mNbNodes; n++)
        std::memcpy(out.data() + n * mB * kDims, padded.data() + n * kMaxBranch * kDims, size_t(mB) * kDims);
    return out;
}

const float* Vocabulary::levelWeights(uint32_t level) const
{
    if (level >= mL) throw Error(kInvalidArg, "level out of range");
    return mWeights.data() + levelBeg(mB, level) * mB;
}

DeviceErrors Vocabulary::takeDeviceErrors() const
{
    DeviceErrors e{};
    RBW_CUDA(cudaMemcpy(&e, mErrors.get(), sizeof(e), cudaMemcpyDeviceToHost));
    RBW_CUDA(cudaMemset(mErrors.get(), 0, sizeof(e)));
    return e;
}

cudaMemPool_t libraryPool()
{
    static cudaMemPool_t pools[64] = {};
    static std::mutex mu;
    int dev = 0;
    RBW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(kUnsupported, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (pools[dev] == nullptr) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        RBW_CUDA(cudaMemPoolCreate(&pools[dev], &props));
        uint64_t keep = ~0ull;
        RBW_CUDA(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return pools[dev];
}

uint32_t Vocabulary::lookup(const uint8_t* devDesc, uint64_t n, uint32_t* devLeaf, LookupAlgo algo,
                            cudaStream_t stream, void* scratch, size_t scratchBytes) const
{
    if (n == 0) return 0;
    if (devDesc == nullptr || devLeaf == nullptr) throw Error(kInvalidArg, "null buffer");
    if (reinterpret_cast<uintptr_t>(devDesc) % 16 != 0)
        throw Error(kInvalidArg, "descriptors must be 16-byte aligned");
    if (mFloat) {
        if (algo == kLookupSimtF32) throw Error(kUnsupported, "the FP32 SIMT lookup reads uint8 centers");
        return lookupFloat(devDesc, n, devLeaf, stream);
    }
    if (algo == kLookupAuto)
        algo = tunedValue(kTuneLookupSchedule, mB, mL, n) == 2 ? kLookupTensorU8Ring : kLookupTensorU8;
    LookupScratch s{};
    if (algo == kLookupSimtF32) {
        s.err = mErrors.as<DeviceErrors>();
        return launchLookup(mTree, devDesc, n, devLeaf, algo, s, stream);
    }
    // TMA row coordinates are signed 32-bit: process at most 2^30 rows per chunk.
    const uint64_t chunk = std::min<uint64_t>(n, 1ull << 30);
    const size_t need = lookupScratchBytes(mB, mL, chunk);
    void* base = scratch;
    bool owned = false;
    if (base == nullptr) {
        RBW_CUDA(cudaMallocFromPoolAsync(&base, need, libraryPool(), stream));
        owned = true;
    } else if (scratchBytes < need) {
        throw Error(kInvalidArg, "lookup scratch too small");
    }
    s = carveLookupScratch(base, mB, mL, chunk);
    s.err = mErrors.as<DeviceErrors>();
    uint32_t kernels = 0;
    for (uint64_t off = 0; off < n; off += chunk) {
        kernels += launchLookup(mTree, devDesc + off * kDims, std::min(chunk, n - off), devLeaf + off, algo, s, stream);
    }
    if (owned) RBW_CUDA(cudaFreeAsync(base, stream));
    return kernels;
}

uint32_t lookupHostPipelined(const Vocabulary& v, const uint8_t* hostDesc, uint64_t n, uint32_t* hostLeaf,
                             LookupAlgo algo)
{
    if (n == 0) return 0;
    if (hostDesc == nullptr || hostLeaf == nullptr) throw Error(kInvalidArg, "null buffer");
    const uint64_t chunk = std::min<uint64_t>(n, 1ull << 20);
    const size_t scratchBytes = lookupScratchBytes(v.branch(), v.levels(), chunk);
    cudaMemPool_t pool = libraryPool();
    cudaStream_t st[2] = {nullptr, nullptr};
    void* dDesc[2] = {nullptr, nullptr};
    void* dLeaf[2] = {nullptr, nullptr};
    void* dScr[2] = {nullptr, nullptr};
    uint32_t kernels = 0;
    auto release = [&] {
        for (int i = 0; i < 2; i++) {
            if (st[i] == nullptr) continue;
            if (dDesc[i]) cudaFreeAsync(dDesc[i], st[i]);
            if (dLeaf[i]) cudaFreeAsync(dLeaf[i], st[i]);
            if (dScr[i]) cudaFreeAsync(dScr[i], st[i]);
            cudaStreamSynchronize(st[i]);
            cudaStreamDestroy(st[i]);
        }
    };
    try {
        for (int i = 0; i < 2; i++) {
            RBW_CUDA(cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking));
            RBW_CUDA(cudaMallocFromPoolAsync(&dDesc[i], chunk * kDims, pool, st[i]));
            RBW_CUDA(cudaMallocFromPoolAsync(&dLeaf[i], chunk * 4, pool, st[i]));
            RBW_CUDA(cudaMallocFromPoolAsync(&dScr[i], scratchBytes, pool, st[i]));
        }
        uint64_t i = 0;
        for (uint64_t off = 0; off < n; off += chunk, i++) {
            const int k = static_cast<int>(i & 1);
            const uint64_t cnt = std::min(chunk, n - off);
            RBW_CUDA(cudaMemcpyAsync(dDesc[k], hostDesc + off * kDims, cnt * kDims, cudaMemcpyHostToDevice, st[k]));
            kernels += v.lookup(static_cast<const uint8_t*>(dDesc[k]), cnt, static_cast<uint32_t*>(dLeaf[k]), algo,
                                st[k], dScr[k], scratchBytes);
            RBW_CUDA(cudaMemcpyAsync(hostLeaf + off, dLeaf[k], cnt * 4, cudaMemcpyDeviceToHost, st[k]));
        }
        for (int k = 0; k < 2; k++) RBW_CUDA(cudaStreamSynchronize(st[k]));
    } catch (...) {
        release();
        throw;
    }
    release();
    return kernels;
}

namespace {
// Build scratch from the library's stream-ordered pool, allocated and freed on the build's
// stream: repeated builds reuse the pool's memory instead of mapping it again, and freeing it
// does not synchronise the device.
class StreamBuffer
{
public:
    StreamBuffer(size_t bytes, cudaStream_t s) : mStream{s}, mBytes{bytes}
    {
        if (bytes) RBW_CUDA(cudaMallocFromPoolAsync(&mPtr, bytes, libraryPool(), s));
    }
    StreamBuffer(const StreamBuffer&) = delete;
    StreamBuffer& operator=(const StreamBuffer&) = delete;
    StreamBuffer(StreamBuffer&& o) noexcept : mPtr{o.mPtr}, mStream{o.mStream}, mBytes{o.mBytes}
    {
        o.mPtr = nullptr;
        o.mBytes = 0;
    }
    StreamBuffer& operator=(StreamBuffer&& o) noexcept
    {
        std::swap(mPtr, o.mPtr);
        std::swap(mStream, o.mStream);
        std::swap(mBytes, o.mBytes);
        return *this;
    }
    ~StreamBuffer()
    {
        if (mPtr) cudaFreeAsync(mPtr, mStream);
    }
    template <typename T>
    T* as() const { return static_cast<T*>(mPtr); }
    void* get() const { return mPtr; }
    size_t bytes() const { return mBytes; }

private:
    void* mPtr = nullptr;
    cudaStream_t mStream = nullptr;
    size_t mBytes = 0;
};
} // namespace

std::unique_ptr<Vocabulary> Vocabulary::build(uint32_t B, uint32_t L, const uint8_t* devDesc, uint32_t nbDesc,
                                              uint32_t nbDoc, const BuildOptions& opts, cudaStream_t stream,
                                              BuildStats* stats)
{
    const auto tStart = std::chrono::steady_clock::now();
    if (B < 2 || B > kMaxBranch) throw Error(kUnsupported, "branch factor must be in [2, 16]");
    if (nbDesc < B) throw Error(kInvalidArg, "Insufficient descriptors"); // Vocabulary.cpp:38-40
    if (nbDoc == 0) throw Error(kInvalidArg, "nbDoc must be positive");   // Vocabulary.cpp:41-43
    if (devDesc == nullptr || reinterpret_cast<uintptr_t>(devDesc) % 16 != 0)
        throw Error(kInvalidArg, "descriptors must be 16-byte aligned device memory");
    if (opts.maxIterations == 0) throw Error(kInvalidArg, "maxIterations must be positive");
    const uint32_t check = std::max(1u, opts.checkInterval);
    std::unique_ptr<Vocabulary> voc{new Vocabulary};
    voc->allocate(B, L);
    const bool fl = opts.floatCenters;
    if (fl) voc->allocateFloat();
    RBW_CUDA(cudaMemsetAsync(voc->mCenters.get(), 0, voc->mCenters.bytes(), stream));
    const uint64_t n = nbDesc;
    const uint64_t maxLevelNodes = ipow(B, L - 1);
    const uint64_t maxChildNodes = ipow(B, L);
    const uint32_t maxTiles128 = static_cast<uint32_t>(n / 128 + maxLevelNodes + 1);
    const uint32_t maxTiles32 = static_cast<uint32_t>(n / 32 + maxLevelNodes + 1);

    const cudaStream_t st = stream;
    StreamBuffer members(n * 4, st), members2(n * 4, st), assign(n, st);
    StreamBuffer nodeCnt(std::max<uint64_t>(maxChildNodes, 1) * 4, st), nodeOff(std::max<uint64_t>(maxChildNodes, 1) * 4, st);
    StreamBuffer childCnt(maxChildNodes * 4, st), childOff(maxChildNodes * 4, st);
    StreamBuffer counts(maxLevelNodes * kMaxBranch * 4, st), sums(maxLevelNodes * kMaxBranch * kDims * 8, st);
    StreamBuffer changed(maxLevelNodes * 4, st), lastChanged(maxLevelNodes * 4, st), small(64, st);
    StreamBuffer picks(maxLevelNodes * B * 4, st), nValid(maxLevelNodes * 4, st);
    StreamBuffer tiles128(uint64_t(maxTiles128) * sizeof(NodeTile), st), tiles32(uint64_t(maxTiles32) * sizeof(NodeTile), st);
    StreamBuffer tileOff(maxLevelNodes * 4, st);
    StreamBuffer scanTmp(scanTempWords(std::max<uint64_t>(uint64_t(B) * maxTiles32, maxLevelNodes)) * 4, st);
    StreamBuffer tileHist(uint64_t(B) * maxTiles32 * 4, st), tileScan(uint64_t(B) * maxTiles32 * 4, st);
    uint32_t* totals = small.as<uint32_t>();
    uint32_t* activeCount = small.as<uint32_t>() + 4;
    // float centers: member |x|^2 sums, per-node inertia, the level's inertia per step, counters
    StreamBuffer qSums(fl ? maxLevelNodes * kMaxBranch * 8 : 0, st), inertiaNode(fl ? maxLevelNodes * 8 : 0, st);
    StreamBuffer inertiaTrace(fl ? uint64_t(opts.maxIterations) * 8 : 0, st), counters(fl ? uint64_t(L) * 16 : 0, st);
    if (fl) {
        RBW_CUDA(cudaMemsetAsync(qSums.get(), 0, qSums.bytes(), stream));
        RBW_CUDA(cudaMemsetAsync(inertiaNode.get(), 0, inertiaNode.bytes(), stream));
        RBW_CUDA(cudaMemsetAsync(counters.get(), 0, counters.bytes(), stream));
    }
    std::vector<double> hostFirst(L, 0.0), hostLast(L, 0.0);
    std::vector<unsigned long long> hostCounters(2 * size_t(L), 0ull);

    iotaKernel<<<blocksFor(n, 256), 256, 0, stream>>>(members.as<uint32_t>(), n);
    RBW_CUDA(cudaGetLastError());
    const uint32_t zero = 0, n32 = nbDesc;
    RBW_CUDA(cudaMemcpyAsync(nodeCnt.get(), &n32, 4, cudaMemcpyHostToDevice, stream));
    RBW_CUDA(cudaMemcpyAsync(nodeOff.get(), &zero, 4, cudaMemcpyHostToDevice, stream));
    RBW_CUDA(cudaMemsetAsync(counts.get(), 0, counts.bytes(), stream));
    RBW_CUDA(cudaMemsetAsync(sums.get(), 0, sums.bytes(), stream));
    RBW_CUDA(cudaMemsetAsync(changed.get(), 0, changed.bytes(), stream));

    // per-node occurrence counts stay on the device until the end (no host copy per level)
    StreamBuffer occDev(voc->mNbNodes * B * 4, st);
    voc->mMasks.assign(voc->mNbNodes, 0u);
    std::mt19937_64 rng{}; // kmeans.cpp:145 (default seed)
    std::vector<uint32_t> hostCnt, hostPicks, hostNValid;
    BuildStats bs{};

    for (uint32_t level = 0; level < L; level++) {
        const uint32_t nbLv = static_cast<uint32_t>(ipow(B, level));
        const uint64_t lb = levelBeg(B, level);
        KMeansLevel lv{};
        lv.B = B;
        lv.nbNodes = nbLv;
        lv.nbMembers = n;
        lv.desc = devDesc;
        lv.members = members.as<uint32_t>();
        lv.nodeOff = nodeOff.as<uint32_t>();
        lv.nodeCnt = nodeCnt.as<uint32_t>();
        lv.centers = voc->mCenters.as<uint8_t>() + lb * kMaxBranch * kDims;
        lv.cnorm = voc->mCnorm.as<int32_t>() + lb * kMaxBranch;
        lv.assign = assign.as<uint8_t>();
        lv.counts = counts.as<uint32_t>();
        lv.sums = sums.as<unsigned long long>();
        lv.changed = changed.as<uint32_t>();
        lv.lastChanged = lastChanged.as<uint32_t>();
        lv.activeCount = activeCount;
        lv.ieeeDivision = opts.ieeeDivision ? 1u : 0u;
        lv.err = voc->mErrors.as<DeviceErrors>();
        KMeansLevelF lvf{};
        if (fl) {
            lvf.base = lv;
            lvf.centers = voc->mCentersF.as<float>() + lb * kMaxBranch * kDims;
            lvf.split = voc->mSplit.as<uint8_t>() + lb * kSplitBytes;
            lvf.cn = voc->mCnF.as<float>() + lb * kMaxBranch;
            lvf.bound = voc->mBound.as<float2>() + lb;
            lvf.q = qSums.as<unsigned long long>();
            lvf.inertiaNode = inertiaNode.as<double>();
            lvf.refined = counters.as<unsigned long long>() + 2 * level;
            lvf.lookupOnly = 0;
        }

        // ---- initial centers
        if (opts.initMode == kInitReference) {
            hostCnt.resize(nbLv);
            RBW_CUDA(cudaMemcpyAsync(hostCnt.data(), nodeCnt.get(), nbLv * 4, cudaMemcpyDeviceToHost, stream));
            RBW_CUDA(cudaStreamSynchronize(stream));
            hostPicks.resize(uint64_t(nbLv) * B);
            for (uint32_t g = 0; g < nbLv; g++) {
                const uint32_t k = referencePick(rng, hostPicks.data() + uint64_t(g) * B, hostCnt[g], B);
                voc->mMasks[lb + g] = k >= 32 ? 0xFFFFFFFFu : ((1u << k) - 1u);
            }
            RBW_CUDA(cudaMemcpyAsync(picks.get(), hostPicks.data(), hostPicks.size() * 4, cudaMemcpyHostToDevice, stream));
            launchInitCenters(lv, picks.as<uint32_t>(), n, stream);
            RBW_CUDA(cudaStreamSynchronize(stream)); // hostPicks is reused next level
        } else if (opts.initMode == kInitKMeansPP) {
            launchKMeansPPInit(lv, opts.seed, level, nValid.as<uint32_t>(), stream);
            hostNValid.resize(nbLv);
            RBW_CUDA(cudaMemcpyAsync(hostNValid.data(), nValid.get(), nbLv * 4, cudaMemcpyDeviceToHost, stream));
            RBW_CUDA(cudaStreamSynchronize(stream));
            for (uint32_t g = 0; g < nbLv; g++) {
                const uint32_t k = hostNValid[g];
                voc->mMasks[lb + g] = k >= 32 ? 0xFFFFFFFFu : ((1u << k) - 1u);
            }
        } else {
            if (opts.injected == nullptr) throw Error(kInvalidArg, "injected initialisation needs indices");
            const uint32_t* inj = opts.injected + lb * B;
            for (uint32_t g = 0; g < nbLv; g++) {
                uint32_t k = 0;
                for (uint32_t b = 0; b < B; b++) {
                    const uint32_t v = inj[uint64_t(g) * B + b];
                    if (v != kInvalidIdx && v >= n) throw Error(kInvalidArg, "injected index out of range");
                    if (v != kInvalidIdx && b == k) k++;
                }
                voc->mMasks[lb + g] = k >= 32 ? 0xFFFFFFFFu : ((1u << k) - 1u);
            }
            RBW_CUDA(cudaMemcpyAsync(picks.get(), inj, uint64_t(nbLv) * B * 4, cudaMemcpyHostToDevice, stream));
            launchInitCentersFromDesc(lv, picks.as<uint32_t>(), n, stream);
            RBW_CUDA(cudaStreamSynchronize(stream));
        }
        if (fl) {
            launchCentersToFloat(lvf, stream);
        } else {
            launchCenterNorms(lv, stream);
        }

        // ---- Lloyd iterations (kmeans.cpp:118-133)
        buildNodeTiles(lv.nodeCnt, lv.nodeOff, nbLv, 128, tileOff.as<uint32_t>(), scanTmp.as<uint32_t>(),
                       tiles128.as<NodeTile>(), maxTiles128, totals, stream);
        RBW_CUDA(cudaMemsetAsync(assign.get(), 0, n, stream)); // fresh (zeroed) assignment memory
        RBW_CUDA(cudaMemsetAsync(lastChanged.get(), 0xFF, uint64_t(nbLv) * 4, stream));
        uint32_t iters = 0;
        for (uint32_t it = 0; it < opts.maxIterations; it++) {
            if (fl) {
                launchAssignF(lvf, tiles128.as<NodeTile>(), totals, maxTiles128, stream);
                RBW_CUDA(cudaMemsetAsync(activeCount, 0, 4, stream));
                launchUpdateF(lvf, stream);
                launchInertiaSum(inertiaNode.as<double>(), nbLv, inertiaTrace.as<double>() + it, stream);
            } else {
                launchAssign(lv, tiles128.as<NodeTile>(), totals, maxTiles128, stream);
                RBW_CUDA(cudaMemsetAsync(activeCount, 0, 4, stream));
                launchUpdate(lv, stream);
            }
            iters = it + 1;
            if ((it + 1) % check == 0 || it + 1 == opts.maxIterations) {
                // the host-side weight array is touched (its pages faulted in) while the device
                // runs the level's first Lloyd steps, not after the last level
                if (voc->mWeights.empty()) voc->mWeights.assign(voc->mNbNodes * B, 0.0f);
                uint32_t active = 0;
                RBW_CUDA(cudaMemcpyAsync(&active, activeCount, 4, cudaMemcpyDeviceToHost, stream));
                RBW_CUDA(cudaStreamSynchronize(stream));
                if (active == 0) break;
            }
        }
        if (level < 16) bs.iterations[level] = iters;
        if (fl) {
            RBW_CUDA(cudaMemcpyAsync(&hostFirst[level], inertiaTrace.get(), 8, cudaMemcpyDeviceToHost, stream));
            RBW_CUDA(cudaMemcpyAsync(&hostLast[level], inertiaTrace.as<double>() + (iters - 1), 8,
                                     cudaMemcpyDeviceToHost, stream));
        }

        // ---- stable regroup into the next level's nodes (Vocabulary.cpp:83-98)
        RegroupScratch rs{tileHist.as<uint32_t>(), tileScan.as<uint32_t>(), scanTmp.as<uint32_t>(),
                          tiles32.as<NodeTile>(), tileOff.as<uint32_t>(), totals, maxTiles32};
        launchRegroup(lv, rs, members2.as<uint32_t>(), childCnt.as<uint32_t>(), childOff.as<uint32_t>(), stream);
        RBW_CUDA(cudaMemcpyAsync(occDev.as<uint32_t>() + lb * B, childCnt.get(), uint64_t(nbLv) * B * 4,
                                 cudaMemcpyDeviceToDevice, stream));
        std::swap(members, members2);
        std::swap(nodeCnt, childCnt);
        std::swap(nodeOff, childOff);
    }
    // the device finishes the tree while the host computes the idf weights
    if (fl) voc->roundFloatCenters(stream);
    voc->finalizeDevice(stream);
    if (fl) {
        RBW_CUDA(cudaMemcpyAsync(hostCounters.data(), counters.get(), hostCounters.size() * 8, cudaMemcpyDeviceToHost,
                                 stream));
    }
    // The counts land in the weights' own storage (one host buffer instead of two) and are
    // turned into weights in place.  Many nodes share a count: the weights of counts below
    // kIdfMemo are computed once (the same expression, so the same float).
    static_assert(sizeof(float) == sizeof(uint32_t), "counts are staged in the weights array");
    voc->mWeights.resize(voc->mNbNodes * B);
    float* w = voc->mWeights.data();
    const size_t nw = voc->mWeights.size();
    RBW_CUDA(cudaMemcpyAsync(w, occDev.get(), nw * 4, cudaMemcpyDeviceToHost, stream));
    // the weights of every count below kIdfMemo, computed once (the same expression, so the same
    // float), while the copy runs
    constexpr uint32_t kIdfMemo = 1u << 12;
    float memo[kIdfMemo];
    for (uint32_t c = 0; c < kIdfMemo; c++) memo[c] = idfWeight(nbDoc, c);
    RBW_CUDA(cudaStreamSynchronize(stream));
    auto weigh = [&](size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; i++) {
            uint32_t c;
            std::memcpy(&c, w + i, 4);
            w[i] = c < kIdfMemo ? memo[c] : idfWeight(nbDoc, c);
        }
    };
    const size_t nThreads = nw >= (size_t(1) << 18) ? 4 : 1;
    std::vector<std::thread> helpers;
    for (size_t k = 1; k < nThreads; k++) helpers.emplace_back(weigh, nw * k / nThreads, nw * (k + 1) / nThreads);
    weigh(0, nw / nThreads);
    for (auto& h : helpers) h.join();
    const DeviceErrors e = voc->takeDeviceErrors();
    if (e.code != 0)
        throw Error(kTimeout, "a bounded device wait gave up during the build (site " + std::to_string(e.where) + ")");
    bs.levels = L;
    for (uint32_t level = 0; level < L && level < 16; level++) {
        bs.inertiaFirst[level] = hostFirst[level];
        bs.inertiaLast[level] = hostLast[level];
        bs.refined[level] = hostCounters[2 * level];
        bs.assignments[level] = hostCounters[2 * level + 1];
    }
    bs.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tStart).count();
    voc->mStats = bs;
    if (stats) *stats = bs;
    return voc;
}

uint32_t Vocabulary::lookupFloat(const uint8_t* devDesc, uint64_t nTotal, uint32_t* devLeaf, cudaStream_t stream) const
{
    // Level by level: the descriptors grouped by node, one split-bf16 assign launch over all the
    // level's nodes (FP64 re-score near ties), then the stable regroup into the children.
    const uint32_t B = mB, L = mL;
    const uint64_t chunk = std::min<uint64_t>(nTotal, 1ull << 27);
    const uint64_t maxLevelNodes = ipow(B, L - 1);
    const uint32_t maxTiles128 = static_cast<uint32_t>(chunk / 128 + maxLevelNodes + 1);
    const uint32_t maxTiles32 = static_cast<uint32_t>(chunk / 32 + maxLevelNodes + 1);
    const cudaStream_t st = stream;
    StreamBuffer members(chunk * 4, st), members2(chunk * 4, st), assign(chunk, st);
    StreamBuffer nodeCnt(maxLevelNodes * 4, st), nodeOff(maxLevelNodes * 4, st);
    StreamBuffer childCnt(maxLevelNodes * 4, st), childOff(maxLevelNodes * 4, st), small(64, st);
    StreamBuffer tiles128(uint64_t(maxTiles128) * sizeof(NodeTile), st);
    StreamBuffer tiles32(uint64_t(maxTiles32) * sizeof(NodeTile), st), tileOff(maxLevelNodes * 4, st);
    StreamBuffer scanTmp(scanTempWords(std::max<uint64_t>(uint64_t(B) * maxTiles32, maxLevelNodes)) * 4, st);
    StreamBuffer tileHist(uint64_t(B) * maxTiles32 * 4, st), tileScan(uint64_t(B) * maxTiles32 * 4, st);
    uint32_t* totals = small.as<uint32_t>();
    uint32_t kernels = 0;
    for (uint64_t off = 0; off < nTotal; off += chunk) {
        const uint32_t n = static_cast<uint32_t>(std::min(chunk, nTotal - off));
        iotaKernel<<<blocksFor(n, 256), 256, 0, stream>>>(members.as<uint32_t>(), n);
        RBW_CUDA(cudaGetLastError());
        const uint32_t zero = 0;
        RBW_CUDA(cudaMemcpyAsync(nodeCnt.get(), &n, 4, cudaMemcpyHostToDevice, stream));
        RBW_CUDA(cudaMemcpyAsync(nodeOff.get(), &zero, 4, cudaMemcpyHostToDevice, stream));
        kernels++;
        for (uint32_t level = 0; level < L; level++) {
            const uint32_t nbLv = static_cast<uint32_t>(ipow(B, level));
            const uint64_t lb = levelBeg(B, level);
            KMeansLevel lv{};
            lv.B = B;
            lv.nbNodes = nbLv;
            lv.nbMembers = n;
            lv.desc = devDesc + off * kDims;
            lv.members = members.as<uint32_t>();
            lv.nodeOff = nodeOff.as<uint32_t>();
            lv.nodeCnt = nodeCnt.as<uint32_t>();
            lv.assign = assign.as<uint8_t>();
            lv.err = mErrors.as<DeviceErrors>();
            KMeansLevelF lvf{};
            lvf.base = lv;
            lvf.centers = mCentersF.as<float>() + lb * kMaxBranch * kDims;
            lvf.split = mSplit.as<uint8_t>() + lb * kSplitBytes;
            lvf.cn = mCnF.as<float>() + lb * kMaxBranch;
            lvf.bound = mBound.as<float2>() + lb;
            lvf.refined = mRefined.as<unsigned long long>();
            lvf.lookupOnly = 1;
            buildNodeTiles(lv.nodeCnt, lv.nodeOff, nbLv, 128, tileOff.as<uint32_t>(), scanTmp.as<uint32_t>(),
                           tiles128.as<NodeTile>(), maxTiles128, totals, stream);
            launchAssignF(lvf, tiles128.as<NodeTile>(), totals, maxTiles128, stream);
            kernels += 7;
            if (level + 1 == L) {
                launchWriteLeaves(lv, tiles128.as<NodeTile>(), totals, maxTiles128, devLeaf + off, stream);
                kernels++;
            } else {
                RegroupScratch rs{tileHist.as<uint32_t>(), tileScan.as<uint32_t>(), scanTmp.as<uint32_t>(),
                                  tiles32.as<NodeTile>(), tileOff.as<uint32_t>(), totals, maxTiles32};
                launchRegroup(lv, rs, members2.as<uint32_t>(), childCnt.as<uint32_t>(), childOff.as<uint32_t>(),
                              stream);
                kernels += 11;
                std::swap(members, members2);
                std::swap(nodeCnt, childCnt);
                std::swap(nodeOff, childOff);
            }
        }
    }
    return kernels;
}

std::vector<uint8_t> Vocabulary::serialize() const
{
    const uint64_t nodes = mNbNodes;
    std::vector<uint8_t> out;
    if (mFloat) {
        // [u32 magic][u32 B][u32 L][f32 centers nodes x B x 128][u32 mask x nodes][f32[B] x nodes]
        const std::vector<float> cf = centersF32Host();
        out.resize(12 + cf.size() * 4 + nodes * 4 + nodes * mB * 4);
        const uint32_t hdr[3] = {kBlobFloatMagic, mB, mL};
        std::memcpy(out.data(), hdr, 12);
        std::memcpy(out.data() + 12, cf.data(), cf.size() * 4);
        std::memcpy(out.data() + 12 + cf.size() * 4, mMasks.data(), nodes * 4);
        std::memcpy(out.data() + 12 + cf.size() * 4 + nodes * 4, mWeights.data(), nodes * mB * 4);
        return out;
    }
    const std::vector<uint8_t> c = centersHost();
    if (mB == 16) {
        // [u32 L][Node: uint32[32 words][16 centers] x nodes][u16 mask x nodes][float[16] x nodes]
        out.resize(4 + nodes * (2048 + 2 + 64));
        std::memcpy(out.data(), &mL, 4);
        uint8_t* nodeBytes = out.data() + 4;
        for (uint64_t n = 0; n < nodes; n++)
            for (uint32_t j = 0; j < 16; j++)
                for (uint32_t w = 0; w < 32; w++)
                    std::memcpy(nodeBytes + n * 2048 + (w * 16 + j) * 4, c.data() + (n * 16 + j) * kDims + w * 4, 4);
        uint8_t* maskBytes = nodeBytes + nodes * 2048;
        for (uint64_t n = 0; n < nodes; n++) {
            const uint16_t m = static_cast<uint16_t>(mMasks[n]);
            std::memcpy(maskBytes + n * 2, &m, 2);
        }
        std::memcpy(maskBytes + nodes * 2, mWeights.data(), nodes * 64);
    } else {
        // [u32 magic][u32 B][u32 L][centers nodes x B x 128][u32 mask x nodes][float[B] x nodes]
        out.resize(12 + nodes * mB * kDims + nodes * 4 + nodes * mB * 4);
        const uint32_t hdr[3] = {kBlobExtMagic, mB, mL};
        std::memcpy(out.data(), hdr, 12);
        std::memcpy(out.data() + 12, c.data(), c.size());
        std::memcpy(out.data() + 12 + c.size(), mMasks.data(), nodes * 4);
        std::memcpy(out.data() + 12 + c.size() + nodes * 4, mWeights.data(), nodes * mB * 4);
    }
    return out;
}

std::unique_ptr<Vocabulary> Vocabulary::deserialize(const uint8_t* blob, size_t size)
{
    if (blob == nullptr || size < 4) throw Error(kInvalidBlob, "invalid blob");
    uint32_t first = 0;
    std::memcpy(&first, blob, 4);
    if (first == kBlobFloatMagic) {
        if (size < 12) throw Error(kInvalidBlob, "invalid blob");
        uint32_t B = 0, L = 0;
        std::memcpy(&B, blob + 4, 4);
        std::memcpy(&L, blob + 8, 4);
        if (B < 2 || B > 16 || L < 1 || L > 8) throw Error(kInvalidBlob, "invalid blob");
        const uint64_t nodes = levelBeg(B, L);
        const uint64_t cBytes = nodes * B * kDims * 4;
        if (size != 12 + cBytes + nodes * 4 + nodes * B * 4) throw Error(kInvalidBlob, "invalid blob");
        std::vector<float> centers(nodes * B * kDims);
        std::vector<uint32_t> masks(nodes);
        std::vector<float> weights(nodes * B);
        std::memcpy(centers.data(), blob + 12, cBytes);
        std::memcpy(masks.data(), blob + 12 + cBytes, nodes * 4);
        std::memcpy(weights.data(), blob + 12 + cBytes + nodes * 4, nodes * B * 4);
        return fromHostF32(B, L, centers.data(), masks.data(), weights.data());
    }
    if (first == kBlobExtMagic) {
        if (size < 12) throw Error(kInvalidBlob, "invalid blob");
        uint32_t B = 0, L = 0;
        std::memcpy(&B, blob + 4, 4);
        std::memcpy(&L, blob + 8, 4);
        if (B < 2 || B > 16 || L < 1 || L > 8) throw Error(kInvalidBlob, "invalid blob");
        const uint64_t nodes = levelBeg(B, L);
        const uint64_t cBytes = nodes * B * kDims;
        if (size != 12 + cBytes + nodes * 4 + nodes * B * 4) throw Error(kInvalidBlob, "invalid blob");
        std::vector<uint32_t> masks(nodes);
        std::vector<float> weights(nodes * B);
        std::memcpy(masks.data(), blob + 12 + cBytes, nodes * 4);
        std::memcpy(weights.data(), blob + 12 + cBytes + nodes * 4, nodes * B * 4);
        return fromHost(B, L, blob + 12, masks.data(), weights.data());
    }
    const uint32_t L = first;
    if (L < 1 || L > 7) throw Error(kInvalidBlob, "invalid blob");
    const uint64_t nodes = levelBeg(16, L);
    if (size != 4 + nodes * (2048 + 2 + 64)) throw Error(kInvalidBlob, "invalid blob"); // Vocabulary.cpp:142-144
    const uint8_t* nodeBytes = blob + 4;
    std::vector<uint8_t> canon(nodes * 16 * kDims);
    for (uint64_t n = 0; n < nodes; n++)
        for (uint32_t j = 0; j < 16; j++)
            for (uint32_t w = 0; w < 32; w++)
                std::memcpy(canon.data() + (n * 16 + j) * kDims + w * 4, nodeBytes + n * 2048 + (w * 16 + j) * 4, 4);
    std::vector<uint32_t> masks(nodes);
    const uint8_t* maskBytes = nodeBytes + nodes * 2048;
    for (uint64_t n = 0; n < nodes; n++) {
        uint16_t m = 0;
        std::memcpy(&m, maskBytes + n * 2, 2);
        masks[n] = m;
    }
    std::vector<float> weights(nodes * 16);
    std::memcpy(weights.data(), maskBytes + nodes * 2, nodes * 64);
    return fromHost(16, L, canon.data(), masks.data(), weights.data());
}

} // namespace rbw
