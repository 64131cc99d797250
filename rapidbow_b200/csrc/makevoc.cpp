// makevoc: builds a vocabulary from a raw descriptor file and writes its blob (the reference's
// main.cpp:27-47, with its constants as defaults and flags to change them).
//
//   makevoc [--docs N] [--levels L] [--branch B] [--init reference|kmeans++] [--seed S]
//           [--iterations N] desc_file voc_file
//
// desc_file holds n x 128 uint8 descriptors back to back; voc_file receives the blob
// (the reference's format for B = 16).  Exit status 0 on success, 1 on bad usage or failure.
#include "rapidbow_b200.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

namespace {

int usage()
{
    std::fprintf(stderr,
                 "usage: makevoc [--docs N] [--levels L] [--branch B] [--init reference|kmeans++] [--seed S]\n"
                 "               [--iterations N] desc_file voc_file\n"
                 "defaults: --docs 527 --levels 5 --branch 16 --init reference --iterations 1000\n");
    return EXIT_FAILURE;
}

bool parseU64(const char* s, uint64_t* v)
{
    char* end = nullptr;
    const unsigned long long x = std::strtoull(s, &end, 10);
    if (end == s || *end != '\0') return false;
    *v = x;
    return true;
}

} // namespace

int main(int argc, char** argv)
{
    uint64_t docs = 527, levels = 5, branch = 16, seed = 0, iterations = 1000; // main.cpp:24-25
    uint32_t initMode = RBW_INIT_REFERENCE;
    std::vector<const char*> files;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto value = [&](uint64_t* v) { return i + 1 < argc && parseU64(argv[++i], v); };
        if (a == "--docs") {
            if (!value(&docs)) return usage();
        } else if (a == "--levels") {
            if (!value(&levels)) return usage();
        } else if (a == "--branch") {
            if (!value(&branch)) return usage();
        } else if (a == "--seed") {
            if (!value(&seed)) return usage();
        } else if (a == "--iterations") {
            if (!value(&iterations)) return usage();
        } else if (a == "--init") {
            if (i + 1 >= argc) return usage();
            const std::string m = argv[++i];
            if (m == "reference") {
                initMode = RBW_INIT_REFERENCE;
            } else if (m == "kmeans++") {
                initMode = RBW_INIT_KMEANSPP;
            } else {
                return usage();
            }
        } else if (a.size() > 1 && a[0] == '-') {
            return usage();
        } else {
            files.push_back(argv[i]);
        }
    }
    if (files.size() != 2) return usage();

    std::ifstream fin(files[0], std::ios::binary | std::ios::ate);
    if (!fin) {
        std::fprintf(stderr, "makevoc: cannot read %s\n", files[0]);
        return EXIT_FAILURE;
    }
    const std::streamsize size = fin.tellg();
    if (size <= 0 || size % 128 != 0 || size / 128 > 0xFFFFFFFFll) {
        std::fprintf(stderr, "makevoc: %s does not hold a whole number of 128-byte descriptors\n", files[0]);
        return EXIT_FAILURE;
    }
    std::vector<char> host(static_cast<size_t>(size));
    fin.seekg(0);
    fin.read(host.data(), size);
    if (!fin) {
        std::fprintf(stderr, "makevoc: short read from %s\n", files[0]);
        return EXIT_FAILURE;
    }

    void* dev = nullptr;
    if (cudaMalloc(&dev, host.size()) != cudaSuccess ||
        cudaMemcpy(dev, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        std::fprintf(stderr, "makevoc: CUDA error: %s\n", cudaGetErrorString(cudaGetLastError()));
        return EXIT_FAILURE;
    }
    rbw_build_options opts;
    rbw_build_options_default(&opts);
    opts.init_mode = initMode;
    opts.seed = seed;
    opts.max_iterations = static_cast<uint32_t>(iterations);
    const rbw_desc_attr sift{RBW_DATA_UINT8, RBW_DIST_L2, 128};
    rbw_vocabulary* voc = nullptr;
    int rc = rbw_voc_build(sift, static_cast<uint32_t>(branch), dev, static_cast<uint32_t>(size / 128),
                           static_cast<uint32_t>(docs), static_cast<uint32_t>(levels), &opts, nullptr, &voc);
    cudaFree(dev);
    if (rc != RBW_OK) {
        std::fprintf(stderr, "makevoc: %s\n", rbw_last_error());
        return EXIT_FAILURE;
    }
    uint64_t bytes = 0;
    rc = rbw_voc_serialize(voc, nullptr, 0, &bytes);
    std::vector<uint8_t> blob(bytes);
    if (rc == RBW_OK) rc = rbw_voc_serialize(voc, blob.data(), blob.size(), &bytes);
    rbw_voc_destroy(voc);
    if (rc != RBW_OK) {
        std::fprintf(stderr, "makevoc: %s\n", rbw_last_error());
        return EXIT_FAILURE;
    }
    std::ofstream fout(files[1], std::ios::binary | std::ios::trunc);
    fout.write(reinterpret_cast<const char*>(blob.data()), static_cast<std::streamsize>(blob.size()));
    if (!fout) {
        std::fprintf(stderr, "makevoc: cannot write %s\n", files[1]);
        return EXIT_FAILURE;
    }
    return EXIT_SUCCESS;
}
