// C++ interface of lowsfer/RapidBoW (RapidBoW.h:28-109), implemented by librapidbow_b200.so on
// top of the C ABI in rapidbow_b200.h.  Existing C++ callers recompile against this header and
// link the library; names, signatures, ownership and exceptions follow the reference:
//   * errors on bad input throw std::runtime_error with the reference's message;
//   * buildVocabulary with unsupported descriptor attributes prints a message and returns an
//     empty pointer (RapidBoW.cpp:37-40);
//   * IVocabulary::lookUp is asynchronous on `stream`, descriptors and leaf indices in device
//     memory; IDataBase takes host leaf indices.
// Differences: branch factors 2..16 are accepted (the reference accepts 16 only), and query
// results with equal scores come back in ascending document order.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime_api.h>
#include <memory>
#include <vector>

#if defined(__GNUC__)
#define RBOW_API __attribute__((visibility("default")))
#else
#define RBOW_API
#endif

namespace rbow {

enum class DataType { kBinary, kUInt8 };

enum class DistanceType { kHamming, kL1, kL2 };

struct DescriptorAttributes {
    DataType dataType;
    DistanceType distanceType;
    size_t nbDims;
};

constexpr DescriptorAttributes SiftAttr{DataType::kUInt8, DistanceType::kL2, 128u};

constexpr inline size_t getDescriptorBytes(DescriptorAttributes attr)
{
    return attr.dataType == DataType::kBinary ? (attr.nbDims + 7) / 8 : attr.nbDims;
}

class RBOW_API IVocabulary
{
public:
    virtual DescriptorAttributes getDescriptorAttributes() const = 0;
    virtual uint32_t getBranchFactor() const = 0;
    virtual uint32_t getNbLevels() const = 0;
    // descriptors and indicesInLeafLevel are device memory
    virtual void lookUp(const void* descriptors, uint32_t nbDesc, uint32_t* indicesInLeafLevel,
                        cudaStream_t stream) const = 0;
    virtual std::vector<std::uint8_t> serialize() const = 0;
    virtual ~IVocabulary();
};

namespace impl {
RBOW_API IVocabulary* buildVocabularyImpl(DescriptorAttributes descAttr, uint32_t branchFactor, const void* devDesc,
                                          uint32_t nbDesc, uint32_t nbDoc, uint32_t nbLevels, cudaStream_t stream);
} // namespace impl

inline std::unique_ptr<IVocabulary> buildVocabulary(DescriptorAttributes descAttr, uint32_t branchFactor,
                                                    const void* devDesc, uint32_t nbDesc, uint32_t nbDoc,
                                                    uint32_t nbLevels, cudaStream_t stream)
{
    return std::unique_ptr<IVocabulary>{
        impl::buildVocabularyImpl(descAttr, branchFactor, devDesc, nbDesc, nbDoc, nbLevels, stream)};
}

RBOW_API std::unique_ptr<IVocabulary> deserializeVocabulary(const std::uint8_t* blob, size_t size);

class RBOW_API IDataBase
{
public:
    virtual const IVocabulary* getVocabulary() const = 0;
    // host leaf indices
    virtual void addDoc(uint32_t idxDoc, const uint32_t* hostIndicesInLeafLevel, uint32_t nbDesc) = 0;
    virtual std::vector<uint32_t> query(const uint32_t* hostIndicesInLeafLevel, uint32_t nbDesc,
                                        uint32_t maxNbResults) const = 0;
    virtual std::vector<uint32_t> queryAndAddDoc(uint32_t idxDoc, const uint32_t* hostIndicesInLeafLevel,
                                                 uint32_t nbDesc, uint32_t maxNbResults) = 0;
    virtual ~IDataBase();
};

// `voc` must come from buildVocabulary or deserializeVocabulary of this library and outlive
// the database.
RBOW_API std::unique_ptr<IDataBase> createDataBase(const IVocabulary* voc);

} // namespace rbow
