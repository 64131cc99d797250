// rbow:: C++ interface (RapidBoW.h of the reference) over this library's C ABI.
#include "RapidBoW.h"
#include "rapidbow_b200.h"

#include <cstdio>
#include <stdexcept>
#include <string>

namespace rbow {

IVocabulary::~IVocabulary() = default;
IDataBase::~IDataBase() = default;

namespace {

[[noreturn]] void fail() { throw std::runtime_error(rbw_last_error()); }

void check(int rc)
{
    if (rc != RBW_OK) fail();
}

class Vocabulary final : public IVocabulary
{
public:
    explicit Vocabulary(rbw_vocabulary* h) : mH{h}
    {
        if (rbw_voc_info(mH, nullptr, &mB, &mL, nullptr) != RBW_OK) {
            rbw_voc_destroy(mH);
            fail();
        }
    }
    ~Vocabulary() override { rbw_voc_destroy(mH); }
    DescriptorAttributes getDescriptorAttributes() const override { return SiftAttr; }
    uint32_t getBranchFactor() const override { return mB; }
    uint32_t getNbLevels() const override { return mL; }
    void lookUp(const void* descriptors, uint32_t nbDesc, uint32_t* indicesInLeafLevel,
                cudaStream_t stream) const override
    {
        check(rbw_voc_lookup(mH, descriptors, nbDesc, indicesInLeafLevel, stream));
    }
    std::vector<std::uint8_t> serialize() const override
    {
        uint64_t size = 0;
        check(rbw_voc_serialize(mH, nullptr, 0, &size));
        std::vector<std::uint8_t> blob(size);
        check(rbw_voc_serialize(mH, blob.data(), blob.size(), &size));
        return blob;
    }
    const rbw_vocabulary* handle() const { return mH; }

private:
    rbw_vocabulary* mH;
    uint32_t mB = 0;
    uint32_t mL = 0;
};

class DataBase final : public IDataBase
{
public:
    explicit DataBase(const Vocabulary* voc) : mVoc{voc} { check(rbw_db_create(voc->handle(), &mH)); }
    ~DataBase() override { rbw_db_destroy(mH); }
    const IVocabulary* getVocabulary() const override { return mVoc; }
    void addDoc(uint32_t idxDoc, const uint32_t* hostIndicesInLeafLevel, uint32_t nbDesc) override
    {
        check(rbw_db_add(mH, idxDoc, hostIndicesInLeafLevel, nbDesc));
    }
    std::vector<uint32_t> query(const uint32_t* hostIndicesInLeafLevel, uint32_t nbDesc,
                                uint32_t maxNbResults) const override
    {
        std::vector<uint32_t> out(maxNbResults);
        uint32_t n = 0;
        check(rbw_db_query(mH, hostIndicesInLeafLevel, nbDesc, maxNbResults, out.data(), nullptr, &n));
        out.resize(n);
        return out;
    }
    std::vector<uint32_t> queryAndAddDoc(uint32_t idxDoc, const uint32_t* hostIndicesInLeafLevel, uint32_t nbDesc,
                                         uint32_t maxNbResults) override
    {
        std::vector<uint32_t> out(maxNbResults);
        uint32_t n = 0;
        check(rbw_db_query_and_add(mH, idxDoc, hostIndicesInLeafLevel, nbDesc, maxNbResults, out.data(), nullptr,
                                   &n));
        out.resize(n);
        return out;
    }

private:
    const Vocabulary* mVoc;
    rbw_database* mH = nullptr;
};

} // namespace

namespace impl {
IVocabulary* buildVocabularyImpl(DescriptorAttributes descAttr, uint32_t branchFactor, const void* devDesc,
                                 uint32_t nbDesc, uint32_t nbDoc, uint32_t nbLevels, cudaStream_t stream)
{
    const rbw_desc_attr attr{static_cast<int32_t>(descAttr.dataType), static_cast<int32_t>(descAttr.distanceType),
                             static_cast<uint64_t>(descAttr.nbDims)};
    rbw_vocabulary* h = nullptr;
    const int rc = rbw_voc_build(attr, branchFactor, devDesc, nbDesc, nbDoc, nbLevels, nullptr, stream, &h);
    if (rc == RBW_ERR_UNSUPPORTED) { // RapidBoW.cpp:37-40: report and return nullptr
        std::fprintf(stderr, "%s\n", rbw_last_error());
        return nullptr;
    }
    check(rc);
    return new Vocabulary(h);
}
} // namespace impl

std::unique_ptr<IVocabulary> deserializeVocabulary(const std::uint8_t* blob, size_t size)
{
    rbw_vocabulary* h = nullptr;
    check(rbw_voc_deserialize(blob, size, &h));
    return std::make_unique<Vocabulary>(h);
}

std::unique_ptr<IDataBase> createDataBase(const IVocabulary* voc)
{
    const auto* v = dynamic_cast<const Vocabulary*>(voc);
    if (v == nullptr) throw std::invalid_argument("createDataBase: vocabulary does not come from this library");
    return std::make_unique<DataBase>(v);
}

} // namespace rbow
