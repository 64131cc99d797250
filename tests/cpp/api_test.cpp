// End-to-end use of the rbow:: C++ interface, as a caller of the reference library writes it
// (the flow of the reference's ApiTest, tests/ApiTests.cpp:36-152, on synthetic images):
// build a vocabulary on the GPU, look every image's descriptors up, add the images to a
// database, and check that each queried image retrieves itself at rank 0.  Also: serialize /
// deserialize gives identical lookups; a duplicate document index throws.
// Exit status 0 = pass.
#include "RapidBoW.h"

#include <cstdio>
#include <cstdlib>
#include <random>
#include <stdexcept>
#include <vector>

#define CHECK(cond)                                                              \
    do {                                                                         \
        if (!(cond)) {                                                           \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
            std::exit(1);                                                        \
        }                                                                        \
    } while (0)

#define CUDA_OK(x) CHECK((x) == cudaSuccess)

int main()
{
    constexpr uint32_t kImages = 40;
    constexpr uint32_t kPerImage = 300;
    constexpr uint32_t kDims = 128;
    std::mt19937_64 rng{3};
    // images are made of descriptors scattered around a few hundred shared cluster means
    std::vector<uint8_t> means(256 * kDims);
    for (auto& m : means) m = static_cast<uint8_t>(rng() % 200);
    std::vector<uint8_t> host(size_t(kImages) * kPerImage * kDims);
    for (uint32_t i = 0; i < kImages * kPerImage; i++) {
        const uint8_t* m = &means[(rng() % 256) * kDims];
        for (uint32_t d = 0; d < kDims; d++) {
            const int v = int(m[d]) + int(rng() % 41) - 20;
            host[size_t(i) * kDims + d] = static_cast<uint8_t>(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    }
    void* devDesc = nullptr;
    uint32_t* devLeaf = nullptr;
    CUDA_OK(cudaMalloc(&devDesc, host.size()));
    CUDA_OK(cudaMalloc(reinterpret_cast<void**>(&devLeaf), size_t(kImages) * kPerImage * 4));
    CUDA_OK(cudaMemcpy(devDesc, host.data(), host.size(), cudaMemcpyHostToDevice));
    cudaStream_t stream;
    CUDA_OK(cudaStreamCreate(&stream));

    // unsupported attributes: message on stderr and an empty pointer (RapidBoW.cpp:37-40)
    const rbow::DescriptorAttributes orb{rbow::DataType::kBinary, rbow::DistanceType::kHamming, 256};
    CHECK(rbow::buildVocabulary(orb, 16, devDesc, kImages * kPerImage, kImages, 3, stream) == nullptr);

    auto voc = rbow::buildVocabulary(rbow::SiftAttr, 16, devDesc, kImages * kPerImage, kImages, 3, stream);
    CHECK(voc != nullptr);
    CHECK(voc->getBranchFactor() == 16 && voc->getNbLevels() == 3);
    CHECK(voc->getDescriptorAttributes().nbDims == 128);

    voc->lookUp(devDesc, kImages * kPerImage, devLeaf, stream);
    std::vector<uint32_t> leaves(size_t(kImages) * kPerImage);
    CUDA_OK(cudaMemcpyAsync(leaves.data(), devLeaf, leaves.size() * 4, cudaMemcpyDeviceToHost, stream));
    CUDA_OK(cudaStreamSynchronize(stream));
    for (const uint32_t l : leaves) CHECK(l < 4096u);

    // serialize -> deserialize -> identical lookups
    const std::vector<uint8_t> blob = voc->serialize();
    auto voc2 = rbow::deserializeVocabulary(blob.data(), blob.size());
    CHECK(voc2->serialize() == blob);
    voc2->lookUp(devDesc, kImages * kPerImage, devLeaf, stream);
    std::vector<uint32_t> leaves2(leaves.size());
    CUDA_OK(cudaMemcpyAsync(leaves2.data(), devLeaf, leaves2.size() * 4, cudaMemcpyDeviceToHost, stream));
    CUDA_OK(cudaStreamSynchronize(stream));
    CHECK(leaves2 == leaves);
    bool threw = false;
    try {
        const uint8_t junk[8] = {1, 2, 3, 4, 5, 6, 7, 8};
        rbow::deserializeVocabulary(junk, sizeof(junk));
    } catch (const std::runtime_error&) {
        threw = true;
    }
    CHECK(threw);

    auto db = rbow::createDataBase(voc.get());
    CHECK(db->getVocabulary() == voc.get());
    for (uint32_t i = 0; i < kImages; i++) db->addDoc(i, &leaves[size_t(i) * kPerImage], kPerImage);
    threw = false;
    try {
        db->addDoc(5, &leaves[0], kPerImage);
    } catch (const std::runtime_error&) {
        threw = true;
    }
    CHECK(threw);
    for (uint32_t i = 0; i < kImages; i++) {
        const auto r = db->query(&leaves[size_t(i) * kPerImage], kPerImage, 10);
        CHECK(!r.empty() && r.size() <= 10);
        CHECK(r[0] == i);
    }
    // queryAndAddDoc: the new image sees the old copy of itself first
    const auto r = db->queryAndAddDoc(1000, &leaves[7 * kPerImage], kPerImage, 4);
    CHECK(!r.empty() && r[0] == 7);
    CHECK(db->query(&leaves[7 * kPerImage], kPerImage, 2).size() == 2);

    db.reset();
    voc2.reset();
    voc.reset();
    CUDA_OK(cudaFree(devDesc));
    CUDA_OK(cudaFree(devLeaf));
    CUDA_OK(cudaStreamDestroy(stream));
    std::printf("api_test: ok\n");
    return 0;
}
