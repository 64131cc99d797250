// Hierarchical k-means training kernels (reference: kmeans.cu, reformatDesc.cu, kmeans.cpp,
// Vocabulary.cpp:66-108).  One grouped launch per Lloyd step covers every node of a tree level.
#pragma once
#include "rbw_common.cuh"

namespace rbw {

// Work item: up to `tileRows` consecutive members of one node.
struct NodeTile {
    uint32_t node;   // in-level node index
    uint32_t start;  // first member position
    uint32_t count;  // members in this tile
    uint32_t first;  // index of the node's first tile (for per-node segmented scans)
};

// Per-level k-means state (device pointers).
struct KMeansLevel {
    uint32_t B;
    uint32_t nbNodes;
    uint64_t nbMembers;
    const uint8_t* desc;        // [nbDesc][128]
    const uint32_t* members;    // [nbMembers] descriptor indices, node segments contiguous
    const uint32_t* nodeOff;    // [nbNodes] first member position of each node
    const uint32_t* nodeCnt;    // [nbNodes]
    uint8_t* centers;           // [nbNodes][16][128] (this level's slice of the tree)
    int32_t* cnorm;             // [nbNodes][16]
    uint8_t* assign;            // [nbMembers]
    uint32_t* counts;           // [nbNodes][16]
    unsigned long long* sums;   // [nbNodes][16][128]
    uint32_t* changed;          // [nbNodes] this iteration
    uint32_t* lastChanged;      // [nbNodes] previous iteration (0 = frozen)
    uint32_t* activeCount;      // [1] nodes whose update ran in the last step
    uint32_t ieeeDivision;      // 0: the reference's fast division, 1: IEEE round-to-nearest
    DeviceErrors* err;          // bounded-wait timeouts of the assign kernel
};

// Exclusive scan helpers (multi-block), tmp needs scanTempWords(n) words.
size_t scanTempWords(uint64_t n);
void exclusiveScanU32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* tmp, cudaStream_t s);

// Tiles of `tileRows` members per node: tileOff = exclusive scan of ceil(cnt/tileRows),
// writes tiles[] and totals[0] = number of tiles.
void buildNodeTiles(const uint32_t* nodeCnt, const uint32_t* nodeOff, uint32_t nbNodes, uint32_t tileRows,
                    uint32_t* tileOff, uint32_t* tmp, NodeTile* tiles, uint32_t maxTiles, uint32_t* totals,
                    cudaStream_t s);

// Initial centers: centers[g][b] = desc[members[nodeOff[g] + pos[g][b]]], or 0xFF bytes when the
// position is past the member array / invalid (reformatDesc.cu:88-96 with kmeans.cpp:179-186).
void launchInitCenters(const KMeansLevel& lv, const uint32_t* pos, uint64_t nbDescTotal, cudaStream_t s);
// Initial centers from descriptor indices (kInvalidIdx -> 0xFF bytes): injected initialisation.
void launchInitCentersFromDesc(const KMeansLevel& lv, const uint32_t* descIdx, uint64_t nbDescTotal, cudaStream_t s);
// Seeded k-means++ over <= 256 sampled members per node; writes centers, cnorm and nValid[g].
void launchKMeansPPInit(const KMeansLevel& lv, uint64_t seed, uint32_t level, uint32_t* nValid, cudaStream_t s);
// |c|^2 for every slot of this level's nodes (padding slots b >= B get kPadNorm).
void launchCenterNorms(const KMeansLevel& lv, cudaStream_t s);

// One assign step over all non-frozen nodes (kmeans.cu:95-300 semantics).
void launchAssign(const KMeansLevel& lv, const NodeTile* tiles, const uint32_t* nTilesDev, uint32_t maxTiles,
                  cudaStream_t s);
// One update step (kmeans.cu:334-375): nodes with changed != 0 get round(sum / count) (fast
// division, as the reference's --use_fast_math build), counts/sums are cleared, lastChanged =
// changed, activeCount = number of nodes updated.
void launchUpdate(const KMeansLevel& lv, cudaStream_t s);

// ------------------------------------------------------------------ float-center mode
// fp32 centers (the FP64 quotient of the exact integer sums, rounded once), distances from the
// tensor core in bf16 with each center split into hi + lo bf16 parts and fp32 accumulation, and
// an FP64 re-score of every member whose best-versus-second margin is within the error bound.
// Per node, `split` holds the MMA B operand: [2 K-blocks of 64 dims][32 rows][128 B] bf16 in the
// 128-byte swizzled K-major layout, rows 0-15 the hi parts and rows 16-31 the lo parts.
constexpr uint32_t kSplitBytes = 2 * 32 * 128;
constexpr float kPadNormF = 3.0e38f; // |c|^2 of padding slots: never the argmin

struct KMeansLevelF {
    KMeansLevel base;             // members, groups, assign, counts, sums, change counters, err
    float* centers;               // [nbNodes][16][128] this level's slice
    uint8_t* split;               // [nbNodes][kSplitBytes]
    float* cn;                    // [nbNodes][16] |c|^2 rounded to fp32 (kPadNormF for padding)
    float2* bound;                // [nbNodes] (max |c|, max |c|^2) over the valid centers
    unsigned long long* q;        // [nbNodes][16] sums of |x|^2 of each center's members
    double* inertiaNode;          // [nbNodes] FP64 inertia of the node's last assignment
    unsigned long long* refined;  // [2] members re-scored in FP64, members assigned (accumulated)
    uint32_t lookupOnly;          // 1: assignment only (lookup through a float tree)
};

// fp32 centers from this level's uint8 initial centers (base.centers), then split, norms, bound.
void launchCentersToFloat(const KMeansLevelF& lv, cudaStream_t s);
// Split, norms and bound of nbNodes nodes of fp32 centers (tree upload / deserialisation).
void launchPrepareFloatNodes(const float* centers, uint8_t* split, float* cn, float2* bound, uint64_t nbNodes,
                             uint32_t B, cudaStream_t s);
// One assign step (build) or one level of a lookup (lookupOnly) over 128-member node tiles.
void launchAssignF(const KMeansLevelF& lv, const NodeTile* tiles, const uint32_t* nTilesDev, uint32_t maxTiles,
                   cudaStream_t s);
// One update step: inertia of the assignment just made, c = float(double(sum) / double(count)).
void launchUpdateF(const KMeansLevelF& lv, cudaStream_t s);
// out[0] = sum of inertiaNode[0, nbNodes) in a fixed order (deterministic).
void launchInertiaSum(const double* inertiaNode, uint32_t nbNodes, double* out, cudaStream_t s);
// Leaf of every member of the last level: leaf[members[i]] = node(i) * B + assign[i].
void launchWriteLeaves(const KMeansLevel& lv, const NodeTile* tiles, const uint32_t* nTilesDev, uint32_t maxTiles,
                       uint32_t* leaf, cudaStream_t s);

// Stable regroup of every node's members by assignment (Vocabulary.cpp:83-98):
// children (g, b) are laid out in order g*B + b; childCnt/childOff have nbNodes*B entries.
struct RegroupScratch {
    uint32_t* tileHist;   // [B][maxTiles]
    uint32_t* tileScan;   // [B][maxTiles]
    uint32_t* scanTmp;
    NodeTile* tiles;      // 32-member tiles
    uint32_t* tileOff;    // [nbNodes]
    uint32_t* totals;     // [2]
    uint32_t maxTiles;
};
void launchRegroup(const KMeansLevel& lv, const RegroupScratch& rs, uint32_t* childMembers, uint32_t* childCnt,
                   uint32_t* childOff, cudaStream_t s);

} // namespace rbw
