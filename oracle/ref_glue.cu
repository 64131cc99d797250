// Test infrastructure only (checker, never product): an extern "C" surface over the
// UNMODIFIED reference sources compiled by oracle/Makefile into oracle/_ref/libref_rbow.so.
// Tests call it through ctypes to compare the product against the reference itself.
//
// CPU-callable: the reference DataBase (DataBase.cpp) over a host-only vocabulary stand-in
//               (the DataBase only needs getNbLevels/getLevelWeights, RapidBoWInternal.h:26-31).
// GPU-only   : reference vocabulary build (Vocabulary.cpp:32-121 via RapidBoW.cpp:26-41),
//               reference lookup kernel (vocTreeLookUp.cu:165-171), and the reference k-means
//               kernels on single tasks (kmeans.cu:302-384, as tests/KmeansAssignCenterTests.cpp
//               drives them).
#include "RapidBoW.h"
#include "RapidBoWInternal.h"
#include "DataBase.h"
#include "Vocabulary.h"
#include "kmeans.h"
#include "vocTreeLookUp.h"
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

namespace {
thread_local std::string gLastError;

template <typename F>
int guarded(F&& f)
{
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        gLastError = e.what();
        return -1;
    }
}

// Host-only IVocabularyInternal: holds nbLevels and the per-node weights array
// (float[levelBeg(L)][16], the layout of Vocabulary::mWeights, Vocabulary.h:86).
class HostWeightsVocabulary : public rbow::IVocabularyInternal
{
public:
    HostWeightsVocabulary(uint32_t nbLevels, const float* weights) : mNbLevels{nbLevels}
    {
        const uint32_t nbNodes = rbow::FullTree<4>::levelBeg(nbLevels);
        mWeights.assign(weights, weights + size_t(nbNodes) * 16);
    }
    rbow::DescriptorAttributes getDescriptorAttributes() const override { return rbow::SiftAttr; }
    uint32_t getBranchFactor() const override { return 16; }
    uint32_t getNbLevels() const override { return mNbLevels; }
    void lookUp(const void*, uint32_t, uint32_t*, cudaStream_t) const override
    {
        throw std::runtime_error("host-only vocabulary");
    }
    std::vector<std::uint8_t> serialize() const override { return {}; }
    const void* getLevelWeights(uint32_t idxLevel) const override
    {
        return &mWeights.at(size_t(rbow::FullTree<4>::levelBeg(idxLevel)) * 16);
    }

private:
    uint32_t mNbLevels;
    std::vector<float> mWeights;
};

// KMeans with configurable iteration cap and check interval (both protected members,
// kmeans.h:113-118).
class KMeansConfigured : public KMeans
{
public:
    KMeansConfigured(const Traits::Descriptor* d, uint32_t n, cudaStream_t s, uint32_t maxIter,
                     uint32_t checkInterval)
        : KMeans{d, n, s}
    {
        mMaxNbIterations = maxIter;
        mConvergenceCheckInterval = checkInterval;
    }
};
} // namespace

extern "C" {

const char* ref_last_error() { return gLastError.c_str(); }

// ---------------------------------------------------------------- CPU: DataBase
void* ref_hostvoc_create(uint32_t nbLevels, const float* weights)
{
    return new HostWeightsVocabulary(nbLevels, weights);
}
void ref_hostvoc_destroy(void* v) { delete static_cast<HostWeightsVocabulary*>(v); }

void* ref_db_create(const void* voc)
{
    return rbow::createDataBase(static_cast<const rbow::IVocabulary*>(voc)).release();
}
void ref_db_destroy(void* db) { delete static_cast<rbow::IDataBase*>(db); }

int ref_db_add(void* db, uint32_t idxDoc, const uint32_t* leaves, uint32_t n)
{
    return guarded([&] { static_cast<rbow::IDataBase*>(db)->addDoc(idxDoc, leaves, n); });
}

int ref_db_query(const void* db, const uint32_t* leaves, uint32_t n, uint32_t k, uint32_t* out,
                 uint32_t* nOut)
{
    return guarded([&] {
        const auto r = static_cast<const rbow::IDataBase*>(db)->query(leaves, n, k);
        std::copy(r.begin(), r.end(), out);
        *nOut = static_cast<uint32_t>(r.size());
    });
}

// Runs `nQueries` concurrent queries over `nThreads` host threads (the DataBase takes a
// shared lock in query, DataBase.cpp:72).  offsets has nQueries+1 entries; out is
// [nQueries][k] with nOut[q] valid entries.  Used for the timed CPU baseline.
int ref_db_query_batch(const void* db, const uint32_t* leaves, const uint64_t* offsets,
                       uint32_t nQueries, uint32_t k, uint32_t* out, uint32_t* nOut,
                       uint32_t nThreads)
{
    return guarded([&] {
        const auto* d = static_cast<const rbow::IDataBase*>(db);
        std::vector<std::thread> pool;
        std::vector<std::string> errors(nThreads);
        for (uint32_t t = 0; t < nThreads; t++) {
            pool.emplace_back([&, t] {
                try {
                    for (uint32_t q = t; q < nQueries; q += nThreads) {
                        const auto r = d->query(leaves + offsets[q],
                                                static_cast<uint32_t>(offsets[q + 1] - offsets[q]), k);
                        std::copy(r.begin(), r.end(), out + size_t(q) * k);
                        nOut[q] = static_cast<uint32_t>(r.size());
                    }
                } catch (const std::exception& e) {
                    errors[t] = e.what();
                }
            });
        }
        for (auto& th : pool) th.join();
        for (const auto& e : errors) {
            if (!e.empty()) throw std::runtime_error(e);
        }
    });
}

// ---------------------------------------------------------------- GPU: vocabulary
// Builds a vocabulary with the reference (fresh thread, so its thread_local init RNG starts
// from the default seed, kmeans.cpp:145) and returns the serialized blob
// (Vocabulary.cpp:175-198).  maxIter == 0 keeps the reference defaults (1000 iterations,
// check interval 4); otherwise the level loop of Vocabulary.cpp:66-99 is re-driven with a
// KMeans whose cap and check interval are set.
int ref_build_vocabulary(const uint8_t* hostDesc, uint32_t nbDesc, uint32_t nbDoc, uint32_t nbLevels,
                         uint32_t maxIter, uint32_t checkInterval, uint8_t** blobOut, uint64_t* blobSize)
{
    int rc = 0;
    std::thread worker([&] {
        rc = guarded([&] {
            auto devDesc = allocCudaMem<uint8_t>(size_t(nbDesc) * 128);
            cudaCheck(cudaMemcpy(devDesc.get(), hostDesc, size_t(nbDesc) * 128, cudaMemcpyHostToDevice));
            std::vector<uint8_t> blob;
            if (maxIter == 0) {
                const auto voc = rbow::buildVocabulary(rbow::SiftAttr, 16, devDesc.get(), nbDesc, nbDoc,
                                                       nbLevels, nullptr);
                blob = voc->serialize();
            } else {
                using Tree = rbow::FullTree<4>;
                using Traits = KMeansTraits;
                const uint32_t nbNodes = Tree::levelBeg(nbLevels);
                auto centers = allocCudaMem<Traits::Centers, CudaMemType::kDevice>(nbNodes);
                auto masks = allocCudaMem<BitSet<16>, CudaMemType::kDevice, true>(nbNodes);
                std::vector<std::vector<uint32_t>> groups{std::vector<uint32_t>(nbDesc)};
                for (uint32_t i = 0; i < nbDesc; i++) groups[0][i] = i;
                std::vector<uint32_t> occ(size_t(nbNodes) * 16, 0u);
                KMeansConfigured km{reinterpret_cast<const Traits::Descriptor*>(devDesc.get()), nbDesc,
                                    nullptr, maxIter, checkInterval};
                for (uint32_t level = 0; level < nbLevels; level++) {
                    const DescGrouping grouping{groups};
                    const uint32_t nbTiles = divUp(grouping.idxEnd(grouping.getNbGrps() - 1u), Traits::tileSize);
                    auto nearest = allocCudaMem<KArray<uint8_t, Traits::tileSize>, CudaMemType::kDevice, true>(nbTiles);
                    km.setGrouping(&grouping, nearest.get(), &centers[Tree::levelBeg(level)],
                                   &masks[Tree::levelBeg(level)]);
                    km.compute(0u, grouping.getNbGrps());
                    std::vector<uint8_t> idx(size_t(Traits::tileSize) * nbTiles);
                    cudaCheck(cudaMemcpy(idx.data(), nearest.get(), idx.size(), cudaMemcpyDeviceToHost));
                    groups.clear();
                    groups.resize(size_t(grouping.getNbGrps()) * 16);
                    for (uint32_t g = 0; g < grouping.getNbGrps(); g++) {
                        for (uint32_t i = grouping.idxBeg(g); i < grouping.idxEnd(g); i++) {
                            groups[size_t(g) * 16 + idx[i]].push_back(grouping.getIndices()[i]);
                        }
                        for (uint32_t b = 0; b < 16; b++) {
                            occ[(size_t(Tree::levelBeg(level)) + g) * 16 + b] =
                                static_cast<uint32_t>(groups[size_t(g) * 16 + b].size());
                        }
                    }
                }
                std::vector<float> w(occ.size());
                for (size_t i = 0; i < occ.size(); i++) {
                    w[i] = occ[i] == 0 ? std::numeric_limits<float>::min()
                                       : std::max(std::numeric_limits<float>::min(),
                                                  std::log(float(nbDoc) / float(occ[i])));
                }
                blob.resize(4 + size_t(nbNodes) * (2048 + 2 + 64));
                std::memcpy(blob.data(), &nbLevels, 4);
                cudaCheck(cudaMemcpy(blob.data() + 4, centers.get(), size_t(nbNodes) * 2048, cudaMemcpyDeviceToHost));
                cudaCheck(cudaMemcpy(blob.data() + 4 + size_t(nbNodes) * 2048, masks.get(), size_t(nbNodes) * 2,
                                     cudaMemcpyDeviceToHost));
                std::memcpy(blob.data() + 4 + size_t(nbNodes) * 2050, w.data(), size_t(nbNodes) * 64);
            }
            *blobSize = blob.size();
            *blobOut = static_cast<uint8_t*>(std::malloc(blob.size()));
            std::memcpy(*blobOut, blob.data(), blob.size());
        });
    });
    worker.join();
    return rc;
}

void ref_free(void* p) { std::free(p); }

// Lookup through the reference API: deserialize (RapidBoW.cpp:43-46) + IVocabulary::lookUp.
int ref_lookup(const uint8_t* blob, uint64_t blobSize, const uint8_t* hostDesc, uint32_t nbDesc,
               uint32_t* hostOut)
{
    return guarded([&] {
        const auto voc = rbow::deserializeVocabulary(blob, blobSize);
        auto devDesc = allocCudaMem<uint8_t>(size_t(nbDesc) * 128 + 16);
        auto devOut = allocCudaMem<uint32_t>(size_t(nbDesc) + 1);
        cudaCheck(cudaMemcpy(devDesc.get(), hostDesc, size_t(nbDesc) * 128, cudaMemcpyHostToDevice));
        voc->lookUp(devDesc.get(), nbDesc, devOut.get(), nullptr);
        cudaCheck(cudaDeviceSynchronize());
        cudaCheck(cudaMemcpy(hostOut, devOut.get(), size_t(nbDesc) * 4, cudaMemcpyDeviceToHost));
    });
}

// Device time of the reference lookup kernel (launchVocTreeLookUp via IVocabulary::lookUp) on
// descriptors already in device memory: `iters` launches bracketed by CUDA events.
int ref_lookup_device_timed(const uint8_t* blob, uint64_t blobSize, const uint8_t* hostDesc, uint32_t nbDesc,
                            uint32_t* hostOut, uint32_t iters, float* msPerLaunch)
{
    return guarded([&] {
        const auto voc = rbow::deserializeVocabulary(blob, blobSize);
        auto devDesc = allocCudaMem<uint8_t>(size_t(nbDesc) * 128 + 16);
        auto devOut = allocCudaMem<uint32_t>(size_t(nbDesc) + 1);
        cudaCheck(cudaMemcpy(devDesc.get(), hostDesc, size_t(nbDesc) * 128, cudaMemcpyHostToDevice));
        voc->lookUp(devDesc.get(), nbDesc, devOut.get(), nullptr);
        cudaEvent_t e0, e1;
        cudaCheck(cudaEventCreate(&e0));
        cudaCheck(cudaEventCreate(&e1));
        cudaCheck(cudaEventRecord(e0, nullptr));
        for (uint32_t i = 0; i < iters; i++) voc->lookUp(devDesc.get(), nbDesc, devOut.get(), nullptr);
        cudaCheck(cudaEventRecord(e1, nullptr));
        cudaCheck(cudaEventSynchronize(e1));
        float ms = 0;
        cudaCheck(cudaEventElapsedTime(&ms, e0, e1));
        *msPerLaunch = ms / float(iters ? iters : 1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaCheck(cudaMemcpy(hostOut, devOut.get(), size_t(nbDesc) * 4, cudaMemcpyDeviceToHost));
    });
}

// One reference assign + (optionally) update on a single k-means task, as
// tests/KmeansAssignCenterTests.cpp:94-105,241-253 drive the kernels.
//   tilesIn : DescTile layout, uint32[nbTiles][32 words][32 desc]
//   centers : Centers layout, uint32[32 words][16 centers]  (in/out when doUpdate)
//   assign  : uint8[nbTiles*32] (in: previous, out: new)
//   counts  : uint32[16], sums: uint32[128][16], nbChanged: uint32
int ref_kmeans_task(const uint32_t* tilesIn, uint32_t nbTiles, uint32_t nbDesc, uint32_t* centers,
                    uint8_t* assign, uint32_t* counts, uint32_t* sums, uint32_t* nbChanged, int doUpdate)
{
    return guarded([&] {
        using Traits = KMeansTraits;
        auto dTiles = allocCudaMem<uint32_t>(size_t(nbTiles) * 1024 + 1);
        auto dCenters = allocCudaMem<uint32_t>(512);
        auto dAssign = allocCudaMem<uint8_t>(size_t(nbTiles) * 32 + 1);
        auto dCounts = allocCudaMem<uint32_t, CudaMemType::kDevice, true>(16);
        auto dSums = allocCudaMem<uint32_t, CudaMemType::kDevice, true>(2048);
        auto dChanged = allocCudaMem<uint32_t, CudaMemType::kDevice, true>(2);
        auto dMask = allocCudaMem<BitSet<16>, CudaMemType::kDevice, true>(1);
        cudaCheck(cudaMemcpy(dTiles.get(), tilesIn, size_t(nbTiles) * 4096, cudaMemcpyHostToDevice));
        cudaCheck(cudaMemcpy(dCenters.get(), centers, 2048, cudaMemcpyHostToDevice));
        cudaCheck(cudaMemcpy(dAssign.get(), assign, size_t(nbTiles) * 32, cudaMemcpyHostToDevice));
        const uint32_t last = 0xFFFFFFFFu;
        cudaCheck(cudaMemcpy(dChanged.get() + 1, &last, 4, cudaMemcpyHostToDevice));
        const uint16_t mask = 0xFFFF;
        cudaCheck(cudaMemcpy(dMask.get(), &mask, 2, cudaMemcpyHostToDevice));
        ArgsKMeansAssignCenter args{reinterpret_cast<const Traits::DescTile*>(dTiles.get()),
                                    nbTiles,
                                    nbDesc,
                                    reinterpret_cast<const Traits::Centers*>(dCenters.get()),
                                    dAssign.get(),
                                    reinterpret_cast<Traits::Counters*>(dCounts.get()),
                                    reinterpret_cast<Traits::GlbCenterAcc*>(dSums.get()),
                                    dChanged.get(),
                                    dChanged.get() + 1,
                                    dMask.get()};
        auto dArgs = allocCudaMem<ArgsKMeansAssignCenter>(1);
        cudaCheck(cudaMemcpy(dArgs.get(), &args, sizeof(args), cudaMemcpyHostToDevice));
        launchAssignCenter(dArgs.get(), 1, nullptr);
        if (doUpdate) {
            launchKMeansUpdateCenters(dArgs.get(), 1, nullptr);
        }
        cudaCheck(cudaDeviceSynchronize());
        cudaCheck(cudaMemcpy(centers, dCenters.get(), 2048, cudaMemcpyDeviceToHost));
        cudaCheck(cudaMemcpy(assign, dAssign.get(), size_t(nbTiles) * 32, cudaMemcpyDeviceToHost));
        cudaCheck(cudaMemcpy(counts, dCounts.get(), 64, cudaMemcpyDeviceToHost));
        cudaCheck(cudaMemcpy(sums, dSums.get(), 8192, cudaMemcpyDeviceToHost));
        cudaCheck(cudaMemcpy(nbChanged, dChanged.get(), 4, cudaMemcpyDeviceToHost));
    });
}

} // extern "C"
