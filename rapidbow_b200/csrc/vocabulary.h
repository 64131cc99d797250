// Vocabulary tree: device-resident centers + host weights (reference: Vocabulary.h:33-87).
#pragma once
#include "lookup.cuh"

#include <cstdint>
#include <memory>
#include <random>
#include <vector>

namespace rbw {

// Owning device buffer.
class DeviceBuffer
{
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t bytes) { reset(bytes); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : mPtr{o.mPtr}, mBytes{o.mBytes}
    {
        o.mPtr = nullptr;
        o.mBytes = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept
    {
        std::swap(mPtr, o.mPtr);
        std::swap(mBytes, o.mBytes);
        return *this;
    }
    ~DeviceBuffer();
    void reset(size_t bytes);
    template <typename T>
    T* as() const { return static_cast<T*>(mPtr); }
    void* get() const { return mPtr; }
    size_t bytes() const { return mBytes; }

private:
    void* mPtr = nullptr;
    size_t mBytes = 0;
};

enum InitMode : uint32_t { kInitReference = 0, kInitKMeansPP = 1, kInitInjected = 2 };

struct BuildOptions {
    uint32_t maxIterations = 1000;  // kmeans.h:118
    uint32_t checkInterval = 4;     // kmeans.h:115
    uint32_t initMode = kInitReference;
    uint64_t seed = 0;
    const uint32_t* injected = nullptr; // host [levelBeg(L)][B] descriptor indices
    bool ieeeDivision = false;          // center update rounding: false = reference (fast-math)
    bool floatCenters = false;          // fp32 centers, split-bf16 distances with FP64 re-score
};

struct BuildStats {
    uint32_t levels = 0;
    uint32_t iterations[16] = {};     // Lloyd steps run per level
    double inertiaFirst[16] = {};     // float centers: FP64 inertia after the level's first step
    double inertiaLast[16] = {};      //                and after its last step
    uint64_t refined[16] = {};        // float centers: assignments re-scored in FP64, all steps
    uint64_t assignments[16] = {};    //                assignments made, all steps
    double seconds = 0;
};

class Vocabulary
{
public:
    // Upload a tree given in the canonical host layout: centers [levelBeg(L)][B][128] uint8,
    // masks [levelBeg(L)] (bit b = valid center), weights [levelBeg(L)][B].
    static std::unique_ptr<Vocabulary> fromHost(uint32_t B, uint32_t L, const uint8_t* centers, const uint32_t* masks,
                                                const float* weights);
    // The same with fp32 centers [levelBeg(L)][B][128]: lookups descend with split-bf16
    // distances and an FP64 re-score near ties.
    static std::unique_ptr<Vocabulary> fromHostF32(uint32_t B, uint32_t L, const float* centers,
                                                   const uint32_t* masks, const float* weights);
    // Hierarchical k-means build on the GPU (Vocabulary.cpp:32-121).  Synchronous.
    static std::unique_ptr<Vocabulary> build(uint32_t B, uint32_t L, const uint8_t* devDesc, uint32_t nbDesc,
                                             uint32_t nbDoc, const BuildOptions& opts, cudaStream_t stream,
                                             BuildStats* stats);
    // Reference blob (Vocabulary.cpp:175-198) for B = 16; a tagged extension otherwise.
    static std::unique_ptr<Vocabulary> deserialize(const uint8_t* blob, size_t size);
    std::vector<uint8_t> serialize() const;

    uint32_t branch() const { return mB; }
    uint32_t levels() const { return mL; }
    uint64_t nbNodes() const { return mNbNodes; }
    const float* levelWeights(uint32_t level) const; // host, [levelSize(level)][B]
    const std::vector<float>& weights() const { return mWeights; }
    const std::vector<uint32_t>& masks() const { return mMasks; }
    // Canonical host copy of the centers ([nbNodes][B][128]); fp32 centers rounded to uint8.
    std::vector<uint8_t> centersHost() const;
    bool floatCenters() const { return mFloat; }
    // fp32 centers ([nbNodes][B][128]) of a float-center vocabulary.
    std::vector<float> centersF32Host() const;
    const DeviceTree& deviceTree() const { return mTree; }
    const BuildStats& buildStats() const { return mStats; }
    // Reads and clears the count of lookup descriptors re-scored in FP64 (float centers).
    uint64_t takeRefinedLookups() const;

    // Stream-ordered lookup; scratch comes from the stream-ordered allocator (or `scratch` if
    // non-null, `scratchBytes` >= lookupScratchBytes).  Returns kernels launched.
    uint32_t lookup(const uint8_t* devDesc, uint64_t n, uint32_t* devLeaf, LookupAlgo algo, cudaStream_t stream,
                    void* scratch = nullptr, size_t scratchBytes = 0) const;
    // Reads (and clears) the device-side error record of this vocabulary's kernels.
    DeviceErrors takeDeviceErrors() const;

private:
    Vocabulary() = default;
    void allocate(uint32_t B, uint32_t L);
    void allocateFloat();
    void finalizeDevice(cudaStream_t stream); // swizzled copy + norms from mCenters
    void roundFloatCenters(cudaStream_t stream); // mCenters = uint8 rounding of mCentersF
    uint32_t lookupFloat(const uint8_t* devDesc, uint64_t n, uint32_t* devLeaf, cudaStream_t stream) const;

    uint32_t mB = 0;
    uint32_t mL = 0;
    uint64_t mNbNodes = 0;
    DeviceBuffer mCenters;   // [nbNodes][16][128]
    DeviceBuffer mCentersSw; // swizzled
    DeviceBuffer mCnorm;     // [nbNodes][16] int32
    DeviceBuffer mErrors;    // DeviceErrors
    std::vector<uint32_t> mMasks;
    std::vector<float> mWeights;
    DeviceTree mTree;
    // float-center vocabularies
    bool mFloat = false;
    DeviceBuffer mCentersF;  // [nbNodes][16][128] float
    DeviceBuffer mSplit;     // [nbNodes][kSplitBytes] bf16 hi/lo MMA operand
    DeviceBuffer mCnF;       // [nbNodes][16] float |c|^2
    DeviceBuffer mBound;     // [nbNodes] float2
    DeviceBuffer mRefined;   // u64: lookup descriptors re-scored in FP64
    BuildStats mStats;
};

// Library-owned stream-ordered memory pool: freed blocks stay cached for the next call.
cudaMemPool_t libraryPool();

// The reference's initial pick of min(space, k) distinct member positions from `rng`, sorted
// and padded with the last pick (kmeans.cpp:141-168); returns the number of distinct picks.
uint32_t referencePick(std::mt19937_64& rng, uint32_t* dst, uint32_t space, uint32_t k);
// idf-like node weight (Vocabulary.cpp:103-108).
float idfWeight(uint32_t nbDoc, uint32_t occ);

// Host-to-host lookup: descriptors are copied in and leaf indices copied back in chunks over
// two streams so transfers overlap the kernels.  Synchronous.  Returns kernels launched.
uint32_t lookupHostPipelined(const Vocabulary& v, const uint8_t* hostDesc, uint64_t n, uint32_t* hostLeaf,
                             LookupAlgo algo);

} // namespace rbw
