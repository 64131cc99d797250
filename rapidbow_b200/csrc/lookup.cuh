// Vocabulary-tree descent (reference: vocTreeLookUp.cu:48-171, Vocabulary.cpp:162-173).
#pragma once
#include "rbw_common.cuh"

namespace rbw {

// Device-resident tree in the layouts the kernels read.  Node slots always hold 16 centers;
// for B < 16 the padding rows are zero and their |c|^2 is kPadNorm (never the argmin).
struct DeviceTree {
    uint32_t B = 0;
    uint32_t L = 0;
    uint64_t nbNodes = 0;
    const uint8_t* centers = nullptr;   // [nbNodes][16][128] row-major (SIMT kernels, update)
    const uint8_t* centersSw = nullptr; // same bytes, 128-byte-swizzled per 8-row atom (MMA B operand)
    const int32_t* cnorm = nullptr;     // [nbNodes][16] exact |c|^2
};

enum LookupAlgo : int {
    kLookupAuto = 0,     // fastest exact path (tensor cores)
    kLookupTensorU8 = 1, // tcgen05 kind::i8, level pairs + counting-sort regroup
    kLookupSimtF32 = 2,  // plain FP32 SIMT kernel (the comparison baseline)
    kLookupTensorU8WarpNode = 3, // as kLookupTensorU8, the node level of each pair by warp-level MMAs
    kLookupTensorU8Ring = 4,     // as kLookupTensorU8, one MMA issuer with a three-slot accumulator ring
    kLookupAlgoLast = kLookupTensorU8Ring,
};

struct LookupStats {
    uint32_t passes;
    uint32_t kernels;
};

// Scratch the tensor-core path needs (all device memory; sizes from lookupScratchBytes).
struct LookupScratch {
    uint32_t* nodeNext = nullptr; // [n]
    uint32_t* perm = nullptr;     // [n]
    uint32_t* bins = nullptr;     // [4 * maxBins + 4] : count | rowOff | tileOff | cursor | total
    void* tiles = nullptr;        // [maxTiles] TileInfo
    uint32_t* ctaHist = nullptr;  // [regroup CTAs][bins] per-CTA bin counts, then their offsets
    DeviceErrors* err = nullptr;
};

size_t lookupScratchBytes(uint32_t B, uint32_t L, uint64_t n);
// Carves `base` (256-B aligned, lookupScratchBytes bytes) into a LookupScratch.
LookupScratch carveLookupScratch(void* base, uint32_t B, uint32_t L, uint64_t n);

// Stream-ordered lookup of n descriptors (16-B aligned device rows of 128 B) into leaf indices.
// Returns the number of kernels launched.
uint32_t launchLookup(const DeviceTree& tree, const uint8_t* desc, uint64_t n, uint32_t* leaf, LookupAlgo algo,
                      const LookupScratch& scratch, cudaStream_t stream);

} // namespace rbw
