// Vocabulary-tree descent kernels (reference semantics: vocTreeLookUp.cu:82-155 -- exact
// squared L2 over 16 centers per node, lowest branch index on ties, idx = idx*B + b).
//
// Two implementations behind launchLookup():
//   * lookupPassTc  : tcgen05 kind::i8 (u8 x u8 -> s32, exact) over level pairs.  A pass takes
//                     the descriptors grouped by their node at level 2p, stages 128-row tiles in
//                     shared memory (a TMA tiled load in input order for the first pass, a 16-byte
//                     cp.async gather through the permutation afterwards), runs one MMA against
//                     the node's 16 centers (level 2p) and one against all of its children's
//                     centers (level 2p+1, N = 16*B), and picks the argmin of |c|^2 - 2 x.c
//                     from tensor memory.  Between passes a device
//                     counting sort (histogram fused into the pass epilogue, scan, scatter)
//                     groups the descriptors by their node at level 2p+2.
//   * lookupSimtF32 : plain FP32 SIMT kernel (one thread per descriptor, 16 fp32 accumulators),
//                     the comparison baseline.  Exact for uint8 data (all sums < 2^24).
#include "lookup.cuh"
#include "timing.h"
#include "tuning.h"

#include <algorithm>
#include <mutex>

namespace rbw {
namespace {

struct TileInfo {
    uint32_t group;
    uint32_t start;
    uint32_t count;
    uint32_t pad;
};

constexpr uint32_t kStages = 8;
constexpr uint32_t kTileRows = 128;
constexpr uint32_t kTileBytes = kTileRows * kDims;    // 16 KB
constexpr uint32_t kNodeBytes = kMaxBranch * kDims;   // 2 KB: one node's 16 centers
constexpr uint32_t kBBlockBytes = kNodeBytes * 17;    // node + up to 16 children
constexpr uint32_t kTeamWarps = 4;                    // epilogue team: one warp per TMEM lane quarter
constexpr uint32_t kIssuer1Warp = 2 + 2 * kTeamWarps;        // second MMA issuer, after the teams
constexpr uint32_t kTcThreads = 32 * (3 + 2 * kTeamWarps); // TMA, two MMA issuers, two epilogue teams
constexpr uint32_t kRingThreads = kTcThreads + 32;          // ring schedule: three MMA issuers
constexpr uint32_t kSmemHistMax = 1024;
constexpr uint32_t kRegroupCtas = 148;                // regroup kernels' CTAs (one per SM on 148 SMs)
// Two accumulator buffers of 256 columns; tile t uses buffer t & 1.  Its level-2p MMA (16
// columns) lands in the first columns of the buffer and is read by the buffer's epilogue team
// before the children MMA of the same tile overwrites the buffer.
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kTmemBuf = 256;
constexpr uint32_t kTileCache = 1024;
// Ring schedule: three 128-column slots for the children accumulators (a tile's children in one
// or two halves of at most 8 children) and eight 16-column node-level entries after them.
constexpr uint32_t kRingSlots = 3;
constexpr uint32_t kSlotCols = 128;
constexpr uint32_t kNodeEntries = 8;
constexpr uint32_t kNodeCol0 = kRingSlots * kSlotCols;
static_assert(kNodeCol0 + 16 * kNodeEntries <= kTmemCols, "ring schedule exceeds tensor memory");
constexpr uint32_t kGatherDepth = 4;                  // gathered tiles in flight (< kStages)
// Row-index ring: iteration i reads slot i % kIdxSlots and queues the copy of tile i + kGatherDepth
// into slot (i + kGatherDepth) % kIdxSlots, which was last read in iteration i - 1 (behind that
// iteration's closing warp barrier).  With kGatherDepth slots the copy would target the slot
// other lanes were still reading, and rows were occasionally gathered from a wrong index.
constexpr uint32_t kIdxSlots = kGatherDepth + 1;

struct TcSmem {
    uint8_t a[kStages][kTileBytes];
    uint8_t b[2][kBBlockBytes];
    uint64_t aFull[kStages];
    uint64_t aEmpty[kStages];
    uint64_t bFull[2];
    uint64_t bEmpty[2];
    uint64_t accA[2];     // level-2p MMA into buffer j complete (one phase per use of j)
    uint64_t aRead[2];    // team j has read the level-2p accumulators of buffer j
    uint64_t accB[2];     // children MMA into buffer j complete
    uint64_t bufFree[2];  // the last reader of buffer j is done with it
    uint64_t lowFree[2];  // team j has read columns [0, 128) of buffer j (two levels only)
    uint64_t mmaDone;
    // ring schedule (lookupPassRing)
    uint64_t nodeAcc[8];  // node-level MMA of tile t complete (entry t % kNodeEntries)
    uint64_t nodeFree[8]; // the team has read entry t % kNodeEntries
    uint64_t slotFull[3]; // children MMA of half n complete (slot n % kRingSlots)
    uint64_t slotFree[3]; // the team has read slot n % kRingSlots
    uint32_t tmemBase;
    uint32_t abortFlag;
    alignas(16) int32_t cn[2][17][16]; // |c|^2 of each B slot: row 0 = node, rows 1.. = children
    uint32_t hist[kSmemHistMax];
    TileInfo tileCache[kTileCache];    // this CTA's tile list (passes after the first)
    alignas(16) int32_t idx[kIdxSlots][kTileRows];    // gather row indices, ring
};
constexpr size_t kTcSmemBytes = sizeof(TcSmem) + 1024;

struct PassParams {
    const uint8_t* desc;     // [nRows][128] descriptors (gathered passes)
    const uint8_t* centersSw;
    const int32_t* cnorm;
    uint32_t B;
    uint32_t twoLevels;
    uint64_t lbA;            // levelBeg of the level the groups live on (2p)
    uint64_t lbB;            // levelBeg(2p + 1)
    uint64_t nRows;
    const uint32_t* perm;    // nullptr for the first pass (rows in input order)
    const TileInfo* tiles;   // nullptr for the first pass
    const uint32_t* nTilesDev;
    uint32_t* out;           // final pass: leaf index per descriptor
    uint32_t* nodeNext;      // other passes: in-level node index at level 2p + 2
    uint32_t* binCount;      // other passes: histogram of nodeNext (nullptr: counted by regroupHist)
    uint32_t nbBins;
    uint32_t isFinal;
    DeviceErrors* err;
};

__device__ __forceinline__ TileInfo getTile(const PassParams& p, uint32_t t)
{
    if (p.tiles == nullptr) {
        const uint64_t s = uint64_t(t) * kTileRows;
        const uint64_t c = p.nRows - s < kTileRows ? p.nRows - s : kTileRows;
        return TileInfo{0u, static_cast<uint32_t>(s), static_cast<uint32_t>(c), 0u};
    }
    return p.tiles[t];
}

// 32 lanes x 64 columns of 32-bit accumulators, and the wait that ties them.
__device__ __forceinline__ void tmemLoad64(uint32_t taddr, uint32_t (&r)[64])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmemWaitTie64(uint32_t (&r)[64])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]), "+r"(r[31]), "+r"(r[32]), "+r"(r[33]), "+r"(r[34]), "+r"(r[35]), "+r"(r[36]), "+r"(r[37]), "+r"(r[38]), "+r"(r[39]), "+r"(r[40]), "+r"(r[41]), "+r"(r[42]), "+r"(r[43]), "+r"(r[44]), "+r"(r[45]), "+r"(r[46]), "+r"(r[47]), "+r"(r[48]), "+r"(r[49]), "+r"(r[50]), "+r"(r[51]), "+r"(r[52]), "+r"(r[53]), "+r"(r[54]), "+r"(r[55]), "+r"(r[56]), "+r"(r[57]), "+r"(r[58]), "+r"(r[59]), "+r"(r[60]), "+r"(r[61]), "+r"(r[62]), "+r"(r[63])
                 :
                 : "memory");
}

// argmin_b (|c_b|^2 - 2 x.c_b), lowest b on ties (vocTreeLookUp.cu:108-125); cnormNode is the
// node's 16 exact |c|^2 values in shared memory.
__device__ __forceinline__ uint32_t argminScores(const uint32_t (&dot)[16], const int32_t* cnormNode)
{
    const int4* cn4 = reinterpret_cast<const int4*>(cnormNode);
    int32_t cn[16];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int4 v = cn4[i];
        cn[4 * i] = v.x;
        cn[4 * i + 1] = v.y;
        cn[4 * i + 2] = v.z;
        cn[4 * i + 3] = v.w;
    }
    int32_t best = cn[0] - 2 * static_cast<int32_t>(dot[0]);
    uint32_t bi = 0;
#pragma unroll
    for (uint32_t b = 1; b < 16; b++) {
        const int32_t s = cn[b] - 2 * static_cast<int32_t>(dot[b]);
        if (s < best) {
            best = s;
            bi = b;
        }
    }
    return bi;
}

// Four 8x8 b16 matrices from shared memory (lanes 8i..8i+7 give the row addresses of matrix i);
// register i of a thread holds row lane/4, bytes 4 (lane % 4) .. + 3 of matrix i.
__device__ __forceinline__ void ldsmX4(uint32_t addr, uint32_t (&r)[4])
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr)
                 : "memory");
}
// d += a (16x32 u8, row-major) * b (32x8 u8, column-major), s32 accumulators (warp-level MMA).
__device__ __forceinline__ void mmaSyncU8(int32_t (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Node-level branch of the warp's 32 tile rows (rows 32 q .. 32 q + 31 of the 128-row tile at
// shared address aBase), with the node's 16 centers at bBase -- both in the 128-byte swizzled
// K-major layout -- by warp-level MMAs (2 row blocks x 2 center blocks x 4 K steps of 32), so the
// tensor memory stays free for the children.  Returns the branch of row 32 q + lane:
// argmin_b (|c_b|^2 - 2 x.c_b), lowest b on ties (vocTreeLookUp.cu:108-125).
__device__ __forceinline__ uint32_t warpNodeArgmin(uint32_t aBase, uint32_t bBase, uint32_t q, uint32_t lane,
                                                   const int32_t* cnormNode)
{
    const uint32_t mi = lane >> 3, r8 = lane & 7u;
    uint32_t res[2][2];
#pragma unroll
    for (uint32_t m = 0; m < 2; m++) {
        // rows 32 q + 16 m .. + 15 against the 16 centers, K in four steps of 32 bytes
        int32_t d[2][4];
#pragma unroll
        for (int n = 0; n < 2; n++)
#pragma unroll
            for (int e = 0; e < 4; e++) d[n][e] = 0;
#pragma unroll
        for (uint32_t kk = 0; kk < 4; kk++) {
            // centers: matrix mi = (centers 8 (mi / 2) .. +7, bytes 16 (mi % 2) of K step kk)
            uint32_t bf[4];
            {
                const uint32_t c = 8u * (mi >> 1) + r8;
                const uint32_t chunk = 2u * kk + (mi & 1u);
                ldsmX4(bBase + c * 128u + ((chunk ^ (c & 7u)) << 4), bf);
            }
            // rows: matrix mi = (rows 16 m + 8 (mi % 2) .. +7, bytes 16 (mi / 2) of K step kk)
            uint32_t af[4];
            {
                const uint32_t row = 32u * q + 16u * m + 8u * (mi & 1u) + r8;
                const uint32_t chunk = 2u * kk + (mi >> 1);
                ldsmX4(aBase + row * 128u + ((chunk ^ (row & 7u)) << 4), af);
            }
            mmaSyncU8(d[0], af, bf[0], bf[1]);
            mmaSyncU8(d[1], af, bf[2], bf[3]);
        }
        // thread holds rows {16 m + lane/4 + 8 h} x centers {8 n + 2 (lane % 4) + e}: d[n][2 h + e]
#pragma unroll
        for (uint32_t h = 0; h < 2; h++) {
            int32_t best = 0x7FFFFFFF;
            uint32_t bi = 0;
#pragma unroll
            for (uint32_t n = 0; n < 2; n++) {
#pragma unroll
                for (uint32_t e = 0; e < 2; e++) {
                    const uint32_t c = 8u * n + 2u * (lane & 3u) + e;
                    const int32_t s = cnormNode[c] - 2 * d[n][2 * h + e];
                    if (s < best) {
                        best = s;
                        bi = c;
                    }
                }
            }
            // the four lanes of a quad hold the row's 16 centers: lowest score, then lowest index
#pragma unroll
            for (uint32_t off = 1; off <= 2; off <<= 1) {
                const int32_t ob = __shfl_xor_sync(0xFFFFFFFFu, best, off);
                const uint32_t oi = __shfl_xor_sync(0xFFFFFFFFu, bi, off);
                if (ob < best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            res[m][h] = bi;
        }
    }
    // row 32 q + lane was computed by quad lane % 8 as (m, h) = (lane / 16, (lane / 8) % 2)
    uint32_t mine = 0;
#pragma unroll
    for (uint32_t m = 0; m < 2; m++)
#pragma unroll
        for (uint32_t h = 0; h < 2; h++) {
            const uint32_t v = __shfl_sync(0xFFFFFFFFu, res[m][h], 4u * (lane & 7u));
            if ((lane >> 4) == m && ((lane >> 3) & 1u) == h) mine = v;
        }
    return mine;
}

// Tile i of this CTA (first pass: computed; later passes: the staged copy of the tile list).
__device__ __forceinline__ TileInfo tileAtSmem(const TcSmem& S, const PassParams& p, uint32_t t0, uint32_t i)
{
    if (p.tiles == nullptr) return getTile(p, t0 + i);
    return i < kTileCache ? S.tileCache[i] : p.tiles[t0 + i];
}
__device__ __forceinline__ bool lastOfGroupSmem(const TcSmem& S, const PassParams& p, uint32_t t0, uint32_t nT,
                                                uint32_t i, uint32_t g)
{
    return i + 1 >= nT || tileAtSmem(S, p, t0, i + 1).group != g;
}
// Writes one row's result: the leaf (last pass) or the next group's node + its histogram count.
__device__ __forceinline__ void emitRow(TcSmem& S, const PassParams& p, bool smemHist, uint32_t orig, uint32_t node)
{
    if (p.isFinal) {
        p.out[orig] = node;
    } else {
        p.nodeNext[orig] = node;
        if (smemHist) {
            atomicAdd(&S.hist[node], 1u);
        } else if (p.binCount != nullptr) {
            atomicAdd(&p.binCount[node], 1u);
        }
    }
}

// ------------------------------------------------------------------ producer warp
// Stages the CTA's tiles [t0, t0 + nT) into the kStages shared-memory slots (arrival on aFull[s],
// waits on aEmpty[s]) and each centre group's block (node + children, bFull / bEmpty).
__device__ __forceinline__ void passProducer(TcSmem& S, const PassParams& p, const CUtensorMap* tmapTile,
                                             uint32_t t0, uint32_t nT, uint32_t lane, volatile uint32_t* abortFlag)
{
    const bool two = p.twoLevels != 0;
    const bool gather = p.perm != nullptr;
    // First pass: one TMA tiled load (128 rows, 128-byte swizzle) per tile.
    // Later passes: the tile's 128 rows are gathered with 16-byte cp.async (lane q copies chunk
    // q % 8 of rows 32 (q / 8) + k) into the same swizzled layout, kGatherDepth tiles in flight.
    // Row indices travel through a shared-memory ring inside the same copy groups: group #i
    // (prologue for i < kGatherDepth, else committed by iteration i - kGatherDepth) carries
    // the indices of tile i and the rows of tile i - kGatherDepth, so wait_group(depth - 1)
    // at the top of iteration i completes both; those rows are then published to the MMA
    // with a proxy fence (generic-proxy writes, async-proxy reader) and an arrival.
    auto copyIdx = [&](uint32_t i) {
        if (i < nT) {
            const TileInfo ti = tileAtSmem(S, p, t0, i);
#pragma unroll
            for (uint32_t j = 0; j < 4; j++) {
                const uint32_t rr = 4 * lane + j;
                cpAsync4(&S.idx[i % kIdxSlots][rr], p.perm + ti.start + (rr < ti.count ? rr : 0u));
            }
        }
    };
    uint32_t published = 0; // tiles [0, published) are visible to the MMA
    auto publishUpTo = [&](uint32_t end) {
        if (published >= end) return;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0)
            for (uint32_t j = published; j < end; j++) mbarArrive(&S.aFull[j % kStages]);
        published = end;
    };
    if (gather) {
        for (uint32_t d = 0; d < kGatherDepth; d++) {
            copyIdx(d);
            cpAsyncCommit();
        }
    }
    uint32_t prevGroup = 0xFFFFFFFFu, slot = 1, slotUses0 = 0, slotUses1 = 0;
    uint32_t issued = 0;
    for (uint32_t i = 0; i < nT; i++) {
        const TileInfo ti = tileAtSmem(S, p, t0, i);
        if (gather) {
            cpAsyncWait<kGatherDepth - 1>();
            if (i >= kGatherDepth) publishUpTo(i - kGatherDepth + 1);
        }
        bool ok = true;
        if (ti.group != prevGroup) {
            // A slot is released only after the MMA and epilogue are done with tile i-2 or
            // earlier, so every gathered tile must be published before waiting for it.
            if (gather) {
                cpAsyncWait<0>();
                publishUpTo(i);
            }
            slot ^= 1u;
            const uint32_t k = slot ? slotUses1++ : slotUses0++;
            if (lane == 0) {
                ok = mbarWait(&S.bEmpty[slot], (k & 1u) ^ 1u, abortFlag, p.err, 10);
                if (ok) {
                    const uint32_t nb = two ? p.B : 0u;
                    mbarArriveExpectTx(&S.bFull[slot], (kNodeBytes + 64u) * (1u + nb));
                    bulkLoad(S.b[slot], p.centersSw + (p.lbA + ti.group) * kNodeBytes, kNodeBytes, &S.bFull[slot]);
                    bulkLoad(&S.cn[slot][0][0], p.cnorm + (p.lbA + ti.group) * kMaxBranch, 64u, &S.bFull[slot]);
                    if (two) {
                        const uint64_t c0 = p.lbB + uint64_t(ti.group) * p.B;
                        bulkLoad(S.b[slot] + kNodeBytes, p.centersSw + c0 * kNodeBytes, kNodeBytes * p.B,
                                 &S.bFull[slot]);
                        bulkLoad(&S.cn[slot][1][0], p.cnorm + c0 * kMaxBranch, 64u * p.B, &S.bFull[slot]);
                    }
                }
            }
            ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
            if (!ok) break;
            prevGroup = ti.group;
        }
        const uint32_t s = i % kStages;
        const uint32_t ph = (i / kStages) & 1u;
        if (lane == 0) {
            ok = mbarWait(&S.aEmpty[s], ph ^ 1u, abortFlag, p.err, 11);
            if (ok && !gather) mbarArriveExpectTx(&S.aFull[s], kTileBytes);
        }
        ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
        if (!ok) break;
        if (!gather) {
            if (lane == 0) tmaLoad2d(S.a[s], tmapTile, 0, static_cast<int32_t>(ti.start), &S.aFull[s]);
        } else {
            // Eight consecutive lanes copy the eight 16-byte chunks of one row, so each
            // instruction moves four whole 128-byte rows (4 lines, not 32).  The indices were
            // written by other lanes' copies: the wait above plus this barrier make them visible.
            __syncwarp();
            // All indices are read before the first copy: the copies are ordered with shared
            // memory accesses, so reads interleaved with them would each wait in turn.
            // Lane group g = lane / 8 copies rows 32 g .. 32 g + 31, whose indices it reads
            // with eight 16-byte loads.
            const int32_t* ring = &S.idx[i % kIdxSlots][0];
            const uint32_t c = lane & 7u;
            uint32_t rowIdx[kTileRows / 4];
#pragma unroll
            for (uint32_t k = 0; k < kTileRows / 16; k++) {
                const int4 v = *reinterpret_cast<const int4*>(ring + 32u * (lane >> 3) + 4u * k);
                rowIdx[4 * k] = static_cast<uint32_t>(v.x);
                rowIdx[4 * k + 1] = static_cast<uint32_t>(v.y);
                rowIdx[4 * k + 2] = static_cast<uint32_t>(v.z);
                rowIdx[4 * k + 3] = static_cast<uint32_t>(v.w);
            }
#pragma unroll
            for (uint32_t k = 0; k < kTileRows / 4; k++) {
                const uint32_t tr = 32u * (lane >> 3) + k; // row within the tile
                cpAsync16(S.a[s] + tr * kDims + ((c ^ (tr & 7u)) << 4), p.desc + uint64_t(rowIdx[k]) * kDims + (c << 4));
            }
            copyIdx(i + kGatherDepth);
            cpAsyncCommit();
        }
        issued = i + 1;
        __syncwarp();
    }
    if (gather) {
        cpAsyncWait<0>();
        publishUpTo(issued);
    } else if (lane == 0) {
        // Drain: every TMA load this warp issued must land before the CTA can exit.
        const uint32_t armed = issued < kStages ? issued : kStages;
        for (uint32_t s = 0; s < armed; s++) {
            const uint32_t last = ((issued - 1 - s) / kStages) * kStages + s; // last i with i % kStages == s
            mbarWait(&S.aFull[s], (last / kStages) & 1u, abortFlag, p.err, 12);
        }
    }
    __syncwarp();
}

// kWarpNode = false: both levels on tcgen05, the node-level MMA and the children MMA of a tile in
// the same TMEM buffer (the children MMA waits until the team has read the node level).
// kWarpNode = true: the epilogue teams take the node level from the shared-memory tile with
// warp-level MMAs (warpNodeArgmin) while the children MMA runs, which is then issued as soon as
// the tile has landed and its buffer is free; a tile slot is released once both its children MMA
// and the team's reads are done.
template <bool kWarpNode>
__global__ void __launch_bounds__(kTcThreads, 1)
    lookupPassTc(const __grid_constant__ CUtensorMap tmapTile, const PassParams p)
{
    extern __shared__ uint8_t smemRaw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    const uint32_t warp = threadIdx.x / 32;
    const uint32_t lane = threadIdx.x % 32;
    const uint32_t T = p.tiles == nullptr ? static_cast<uint32_t>((p.nRows + kTileRows - 1) / kTileRows)
                                          : *p.nTilesDev;
    const uint32_t t0 = static_cast<uint32_t>(uint64_t(T) * blockIdx.x / gridDim.x);
    const uint32_t t1 = static_cast<uint32_t>(uint64_t(T) * (blockIdx.x + 1) / gridDim.x);
    const uint32_t nT = t1 - t0;
    const bool smemHist = !p.isFinal && p.binCount != nullptr && p.nbBins <= kSmemHistMax;
    const bool two = p.twoLevels != 0;
    const bool gather = p.perm != nullptr;
    volatile uint32_t* abortFlag = &S.abortFlag;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < kStages; s++) {
            mbarInit(&S.aFull[s], 1);
            // kWarpNode: the children MMA's commit (two levels) and the four warps of the team
            mbarInit(&S.aEmpty[s], kWarpNode ? (two ? 1u : 0u) + kTeamWarps : 1u);
        }
        for (uint32_t j = 0; j < 2; j++) {
            mbarInit(&S.bFull[j], 1);
            mbarInit(&S.bEmpty[j], 2 + 2 * kTeamWarps); // both MMA issuers + both epilogue teams
            mbarInit(&S.accA[j], 1);
            mbarInit(&S.aRead[j], kTeamWarps);
            mbarInit(&S.accB[j], 1);
            mbarInit(&S.bufFree[j], kTeamWarps);
            mbarInit(&S.lowFree[j], kTeamWarps);
        }
        mbarInit(&S.mmaDone, 2);
        S.abortFlag = 0;
        fenceMbarInit();
    }
    if (smemHist) {
        for (uint32_t i = threadIdx.x; i < p.nbBins; i += blockDim.x) S.hist[i] = 0;
    }
    if (p.tiles != nullptr) {
        const uint32_t m = nT < kTileCache ? nT : kTileCache;
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) S.tileCache[i] = p.tiles[t0 + i];
    }
    if (warp == 0) {
        tmemAlloc(&S.tmemBase, kTmemCols);
        tmemRelinquish();
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = S.tmemBase;
    if (nT > 0 && warp == 0) {
        passProducer(S, p, &tmapTile, t0, nT, lane, abortFlag);
    } else if (nT > 0 && (warp == 1 || warp == kIssuer1Warp)) {
        // ------------------------------------------------------------ MMA issuers (one thread each)
        // Issuer j (warp 1 for j = 0, warp kIssuer1Warp for j = 1) issues the MMAs of the tiles
        // t with t & 1 == j, which accumulate in TMEM buffer j (columns [256 j, 256 j + 256)):
        // a(t) (level 2p, 16 columns) needs only the buffer's first 16 columns, which epilogue
        // team j releases after the first 128-column load of tile t-2, so the level-2p MMA of
        // tile t overlaps the rest of that read; b(t) (children, 16 B columns) waits for the
        // whole buffer and for the team to have read a(t).  One level: a(t) only, released after
        // the team's read.  Two issuers let one buffer's MMAs go while the other's thread
        // waits; commits track only the committing thread's MMAs, so each buffer's barriers see
        // exactly its own tiles.  Both issuers pass every tile and commit once per centre group
        // on the producer's "centre block free" barrier.
        if (lane == 0) {
            const uint32_t jm = warp == 1 ? 0u : 1u;
            const uint32_t idescA = idescU8(16);
            const uint32_t idescB = idescU8(16 * p.B);
            uint32_t prevGroup = 0xFFFFFFFFu, slot = 1, uses0 = 0, uses1 = 0;
            bool ok = true;
            for (uint32_t t = 0; ok && t < nT; t++) {
                const TileInfo ti = tileAtSmem(S, p, t0, t);
                if (ti.group != prevGroup) {
                    slot ^= 1u;
                    const uint32_t u = slot ? uses1++ : uses0++;
                    if (!mbarWait(&S.bFull[slot], u & 1u, abortFlag, p.err, 20)) break;
                    prevGroup = ti.group;
                }
                if constexpr (kWarpNode) {
                    // children only: as soon as the tile has landed and team j has read the
                    // buffer's previous tile
                    if ((t & 1u) == jm && two) {
                        const uint32_t s = t % kStages;
                        if (!mbarWait(&S.aFull[s], (t / kStages) & 1u, abortFlag, p.err, 21)) break;
                        if (t >= 2 && !mbarWait(&S.bufFree[jm], ((t >> 1) - 1u) & 1u, abortFlag, p.err, 25)) break;
                        tcFenceAfter();
                        const uint32_t aBase = smemAddr(S.a[s]);
                        const uint32_t bBase = smemAddr(S.b[slot]);
#pragma unroll
                        for (uint32_t q4 = 0; q4 < 4; q4++) {
                            mmaU8(tmem + kTmemBuf * jm, smemDescSw128(aBase + 32u * q4),
                                  smemDescSw128(bBase + kNodeBytes + 32u * q4), idescB, q4 > 0 ? 1u : 0u);
                        }
                        mmaCommit(&S.accB[jm]);
                        mmaCommit(&S.aEmpty[s]);
                    }
                } else if ((t & 1u) == jm) {
                    const uint32_t j = jm;
                    const uint32_t s = t % kStages;
                    if (!mbarWait(&S.aFull[s], (t / kStages) & 1u, abortFlag, p.err, 21)) break;
                    if (t >= 2 && !mbarWait(two ? &S.lowFree[j] : &S.bufFree[j], ((t >> 1) - 1u) & 1u, abortFlag,
                                            p.err, 22))
                        break;
                    tcFenceAfter();
                    const uint32_t aBase = smemAddr(S.a[s]);
                    const uint32_t bBase = smemAddr(S.b[slot]);
#pragma unroll
                    for (uint32_t q4 = 0; q4 < 4; q4++) {
                        mmaU8(tmem + kTmemBuf * j, smemDescSw128(aBase + 32u * q4),
                              smemDescSw128(bBase + 32u * q4), idescA, q4 > 0 ? 1u : 0u);
                    }
                    mmaCommit(&S.accA[j]);
                    if (two) {
                        if (!mbarWait(&S.aRead[j], (t >> 1) & 1u, abortFlag, p.err, 23)) break;
                        if (t >= 2 && !mbarWait(&S.bufFree[j], ((t >> 1) - 1u) & 1u, abortFlag, p.err, 25)) break;
                        tcFenceAfter();
#pragma unroll
                        for (uint32_t q4 = 0; q4 < 4; q4++) {
                            mmaU8(tmem + kTmemBuf * j, smemDescSw128(aBase + 32u * q4),
                                  smemDescSw128(bBase + kNodeBytes + 32u * q4), idescB, q4 > 0 ? 1u : 0u);
                        }
                        mmaCommit(&S.accB[j]);
                    }
                    mmaCommit(&S.aEmpty[s]);
                }
                if (lastOfGroupSmem(S, p, t0, nT, t, ti.group)) mmaCommit(&S.bEmpty[slot]);
            }
            mmaCommit(&S.mmaDone);
            mbarWait(&S.mmaDone, 0, abortFlag, p.err, 24);
        }
        __syncwarp();
    } else if (nT > 0 && warp >= 2 && warp < 2 + 2 * kTeamWarps) {
        // ------------------------------------------------------------ epilogue teams
        // Team j (warps 2 + 4 j .. 5 + 4 j, one per TMEM lane quarter; each thread owns one tile
        // row) serves buffer j: the tiles t with t & 1 == j.  Per tile it reads the level-2p
        // accumulators and picks the branch (releasing them to the children MMA), then reads the
        // row's 16 * B children columns in 64-column loads -- releasing the first 128
        // columns, where the next level-2p MMA of the buffer lands, after the first load and the
        // buffer after the second -- and keeps the 16 columns of the chosen child.  The branch
        // stays in a register.  With one level the team releases the buffer after the level-2p
        // read.  Each team passes every tile so that both arrive once per centre group on bEmpty.
        const uint32_t team = (warp - 2u) / kTeamWarps;
        const uint32_t q = warp & 3u;
        const uint32_t row = q * 32u + lane;
        const uint32_t tRow = tmem + ((q * 32u) << 16);
        uint32_t prevGroup = 0xFFFFFFFFu, slot = 1, uses0 = 0, uses1 = 0;
        for (uint32_t t = 0; t < nT; t++) {
            const uint32_t j = t & 1u;
            const TileInfo ti = tileAtSmem(S, p, t0, t);
            if (ti.group != prevGroup) {
                // Wait for the group's centre block even when this team has no tile in it: the
                // team's arrival on bEmpty for this group must not come before the block was
                // loaded, or it would count toward the slot's previous group and free that
                // block while the other team still reads it.
                slot ^= 1u;
                const uint32_t u = slot ? uses1++ : uses0++;
                if (!mbarWait(&S.bFull[slot], u & 1u, abortFlag, p.err, 33)) break;
                prevGroup = ti.group;
            }
            if (j == team) {
                const uint32_t orig = row < ti.count ? (gather ? __ldg(p.perm + ti.start + row) : ti.start + row) : 0u;
                const uint32_t base = tRow + kTmemBuf * j;
                uint32_t b;
                if constexpr (kWarpNode) {
                    // node level from the shared-memory tile (warp-level MMAs), while the
                    // children MMA of the same tile runs on the tensor core
                    const uint32_t s = t % kStages;
                    if (!mbarWait(&S.aFull[s], (t / kStages) & 1u, abortFlag, p.err, 34)) break;
                    b = warpNodeArgmin(smemAddr(S.a[s]), smemAddr(S.b[slot]), q, lane, &S.cn[slot][0][0]);
                    __syncwarp();
                    if (lane == 0) mbarArrive(&S.aEmpty[s]); // this warp is done reading the tile
                } else {
                    if (!mbarWait(&S.accA[j], (t >> 1) & 1u, abortFlag, p.err, 30)) break;
                    tcFenceAfter();
                    {
                        uint32_t r[16];
                        tmemLoad16(base, r);
                        tmemWaitTie(r);
                        b = argminScores(r, &S.cn[slot][0][0]);
                    }
                    tcFenceBefore();
                    __syncwarp();
                    if (lane == 0) mbarArrive(two ? &S.aRead[j] : &S.bufFree[j]);
                }
                if (!two) {
                    if (row < ti.count) emitRow(S, p, smemHist, orig, ti.group * p.B + b);
                } else {
                    if (!mbarWait(&S.accB[j], (t >> 1) & 1u, abortFlag, p.err, 31)) break;
                    tcFenceAfter();
                    uint32_t sel[16];
#pragma unroll
                    for (int i = 0; i < 16; i++) sel[i] = 0;
                    // children 4 h .. 4 h + 3 are columns [64 h, 64 h + 64)
                    auto pick = [&](uint32_t h) {
                        uint32_t r[64];
                        tmemLoad64(base + 64u * h, r);
                        tmemWaitTie64(r);
#pragma unroll
                        for (uint32_t k = 0; k < 4; k++)
#pragma unroll
                            for (int i = 0; i < 16; i++) sel[i] = b == 4 * h + k ? r[16 * k + i] : sel[i];
                    };
                    pick(0);
                    pick(1);
                    if constexpr (!kWarpNode) {
                        // columns [0, 128) have been read: the level-2p MMA of tile t + 2 may start
                        tcFenceBefore();
                        __syncwarp();
                        if (lane == 0) mbarArrive(&S.lowFree[j]);
                    }
                    if (p.B > 8) {
                        pick(2);
                        pick(3);
                    }
                    // the accumulators are in registers: the buffer can take tile t + 2
                    tcFenceBefore();
                    __syncwarp();
                    if (lane == 0) mbarArrive(&S.bufFree[j]);
                    if (row < ti.count) {
                        const uint64_t child = uint64_t(ti.group) * p.B + b; // in-level index at level 2p+1
                        const uint32_t b2 = argminScores(sel, &S.cn[slot][1 + b][0]);
                        emitRow(S, p, smemHist, orig, static_cast<uint32_t>(child * p.B + b2));
                    }
                }
            }
            if (lastOfGroupSmem(S, p, t0, nT, t, ti.group)) {
                __syncwarp();
                if (lane == 0) mbarArrive(&S.bEmpty[slot]);
            }
        }
    }

    tcFenceBefore();
    __syncthreads();
    if (smemHist) {
        for (uint32_t i = threadIdx.x; i < p.nbBins; i += blockDim.x) {
            const uint32_t v = S.hist[i];
            if (v) atomicAdd(&p.binCount[i], v);
        }
    }
    if (warp == 0) {
        tcFenceAfter();
        tmemDealloc(tmem, kTmemCols);
    }
}

// Ring schedule.  Three threads issue the MMAs, each in tile order: warp 1 the node-level MMA
// of tile t into node entry t % kNodeEntries; warps 10 and 11 the tile's children in halves
// (children [0, c0) and [c0, B), c0 = ceil(B / 2); one half when B <= 8) into ring slots
// n % kRingSlots, n = the running half index.  No children MMA waits for a node-level read:
// the children accumulators never share columns with the node level, so the tensor pipe runs
// the halves back to back while the teams read earlier slots.  Half n waits only until half
// n - kRingSlots has been read; node entry t until tile t - kNodeEntries's entry has been read.
// Team t & 1 reads the node level, picks the branch b, then reads the halves (64-column loads)
// and keeps the 16 columns of child b.  Every issuer commits its own MMAs (a commit tracks the
// committing thread's MMAs only) to the tile's stage and the group's centre block barriers.
__global__ void __launch_bounds__(kRingThreads, 1)
    lookupPassRing(const __grid_constant__ CUtensorMap tmapTile, const PassParams p)
{
    extern __shared__ uint8_t smemRaw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    const uint32_t warp = threadIdx.x / 32;
    const uint32_t lane = threadIdx.x % 32;
    const uint32_t T = p.tiles == nullptr ? static_cast<uint32_t>((p.nRows + kTileRows - 1) / kTileRows)
                                          : *p.nTilesDev;
    const uint32_t t0 = static_cast<uint32_t>(uint64_t(T) * blockIdx.x / gridDim.x);
    const uint32_t t1 = static_cast<uint32_t>(uint64_t(T) * (blockIdx.x + 1) / gridDim.x);
    const uint32_t nT = t1 - t0;
    const bool smemHist = !p.isFinal && p.binCount != nullptr && p.nbBins <= kSmemHistMax;
    const bool two = p.twoLevels != 0;
    const uint32_t nh = two ? (p.B > 8 ? 2u : 1u) : 0u;   // children halves per tile
    const uint32_t c0 = nh == 2 ? (p.B + 1) / 2 : p.B;     // children in the first half
    const uint32_t issuers = 1 + nh;
    volatile uint32_t* abortFlag = &S.abortFlag;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < kStages; s++) {
            mbarInit(&S.aFull[s], 1);
            mbarInit(&S.aEmpty[s], issuers);
        }
        for (uint32_t j = 0; j < 2; j++) {
            mbarInit(&S.bFull[j], 1);
            mbarInit(&S.bEmpty[j], issuers + 2 * kTeamWarps); // the issuers + both epilogue teams
        }
        for (uint32_t e = 0; e < kNodeEntries; e++) {
            mbarInit(&S.nodeAcc[e], 1);
            mbarInit(&S.nodeFree[e], kTeamWarps);
        }
        for (uint32_t k = 0; k < kRingSlots; k++) {
            mbarInit(&S.slotFull[k], 1);
            mbarInit(&S.slotFree[k], kTeamWarps);
        }
        mbarInit(&S.mmaDone, issuers);
        S.abortFlag = 0;
        fenceMbarInit();
    }
    if (smemHist) {
        for (uint32_t i = threadIdx.x; i < p.nbBins; i += blockDim.x) S.hist[i] = 0;
    }
    if (p.tiles != nullptr) {
        const uint32_t m = nT < kTileCache ? nT : kTileCache;
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) S.tileCache[i] = p.tiles[t0 + i];
    }
    if (warp == 0) {
        tmemAlloc(&S.tmemBase, kTmemCols);
        tmemRelinquish();
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = S.tmemBase;
    // issuer role: 0 node level (warp 1), 1 + h children half h (warps 10 and 11)
    const uint32_t role = warp == 1 ? 0u : warp == kIssuer1Warp ? 1u : warp == kIssuer1Warp + 1 ? 2u : 99u;
    if (nT > 0 && warp == 0) {
        passProducer(S, p, &tmapTile, t0, nT, lane, abortFlag);
    } else if (nT > 0 && role < issuers) {
        // ------------------------------------------------------------ MMA issuers (one thread each)
        if (lane == 0) {
            const uint32_t h = role - 1u;                    // children half (roles 1, 2)
            const uint32_t cb = h ? c0 : 0u;
            const uint32_t cnt = h ? p.B - c0 : c0;
            const uint32_t idesc = role == 0 ? idescU8(16) : idescU8(16u * cnt);
            uint32_t prevGroup = 0xFFFFFFFFu, slot = 1, uses0 = 0, uses1 = 0;
            for (uint32_t t = 0; t < nT; t++) {
                const TileInfo ti = tileAtSmem(S, p, t0, t);
                if (ti.group != prevGroup) {
                    slot ^= 1u;
                    const uint32_t u = slot ? uses1++ : uses0++;
                    if (!mbarWait(&S.bFull[slot], u & 1u, abortFlag, p.err, 40)) break;
                    prevGroup = ti.group;
                }
                const uint32_t s = t % kStages;
                if (!mbarWait(&S.aFull[s], (t / kStages) & 1u, abortFlag, p.err, 41)) break;
                const uint32_t aBase = smemAddr(S.a[s]);
                const uint32_t bBase = smemAddr(S.b[slot]);
                if (role == 0) {
                    const uint32_t e = t % kNodeEntries;
                    if (t >= kNodeEntries &&
                        !mbarWait(&S.nodeFree[e], ((t / kNodeEntries) - 1u) & 1u, abortFlag, p.err, 42))
                        break;
                    tcFenceAfter();
#pragma unroll
                    for (uint32_t q4 = 0; q4 < 4; q4++) {
                        mmaU8(tmem + kNodeCol0 + 16u * e, smemDescSw128(aBase + 32u * q4),
                              smemDescSw128(bBase + 32u * q4), idesc, q4 > 0 ? 1u : 0u);
                    }
                    mmaCommit(&S.nodeAcc[e]);
                } else {
                    const uint32_t n = t * nh + h;
                    const uint32_t k = n % kRingSlots;
                    if (n >= kRingSlots &&
                        !mbarWait(&S.slotFree[k], ((n / kRingSlots) - 1u) & 1u, abortFlag, p.err, 43))
                        break;
                    tcFenceAfter();
                    const uint32_t cBase = bBase + kNodeBytes * (1u + cb);
#pragma unroll
                    for (uint32_t q4 = 0; q4 < 4; q4++) {
                        mmaU8(tmem + kSlotCols * k, smemDescSw128(aBase + 32u * q4),
                              smemDescSw128(cBase + 32u * q4), idesc, q4 > 0 ? 1u : 0u);
                    }
                    mmaCommit(&S.slotFull[k]);
                }
                mmaCommit(&S.aEmpty[s]); // the stage is free once every issuer's MMAs on it are done
                if (lastOfGroupSmem(S, p, t0, nT, t, ti.group)) mmaCommit(&S.bEmpty[slot]);
            }
            mmaCommit(&S.mmaDone);
            mbarWait(&S.mmaDone, 0, abortFlag, p.err, 44);
        }
        __syncwarp();
    } else if (nT > 0 && warp >= 2 && warp < 2 + 2 * kTeamWarps) {
        // ------------------------------------------------------------ epilogue teams
        const uint32_t team = (warp - 2u) / kTeamWarps;
        const uint32_t q = warp & 3u;
        const uint32_t row = q * 32u + lane;
        const uint32_t tRow = tmem + ((q * 32u) << 16);
        const bool gather = p.perm != nullptr;
        uint32_t prevGroup = 0xFFFFFFFFu, slot = 1, uses0 = 0, uses1 = 0;
        for (uint32_t t = 0; t < nT; t++) {
            const TileInfo ti = tileAtSmem(S, p, t0, t);
            if (ti.group != prevGroup) {
                // every team waits for every group's block (see lookupPassTc)
                slot ^= 1u;
                const uint32_t u = slot ? uses1++ : uses0++;
                if (!mbarWait(&S.bFull[slot], u & 1u, abortFlag, p.err, 50)) break;
                prevGroup = ti.group;
            }
            if ((t & 1u) == team) {
                const uint32_t orig = row < ti.count ? (gather ? __ldg(p.perm + ti.start + row) : ti.start + row) : 0u;
                const uint32_t e = t % kNodeEntries;
                if (!mbarWait(&S.nodeAcc[e], (t / kNodeEntries) & 1u, abortFlag, p.err, 51)) break;
                tcFenceAfter();
                uint32_t b;
                {
                    uint32_t r[16];
                    tmemLoad16(tRow + kNodeCol0 + 16u * e, r);
                    tmemWaitTie(r);
                    b = argminScores(r, &S.cn[slot][0][0]);
                }
                tcFenceBefore();
                __syncwarp();
                if (lane == 0) mbarArrive(&S.nodeFree[e]);
                if (!two) {
                    if (row < ti.count) emitRow(S, p, smemHist, orig, ti.group * p.B + b);
                } else {
                    uint32_t sel[16];
#pragma unroll
                    for (int i = 0; i < 16; i++) sel[i] = 0;
                    bool ok = true;
                    for (uint32_t h = 0; h < nh; h++) {
                        const uint32_t n = t * nh + h;
                        const uint32_t k = n % kRingSlots;
                        if (!mbarWait(&S.slotFull[k], (n / kRingSlots) & 1u, abortFlag, p.err, 52)) {
                            ok = false;
                            break;
                        }
                        tcFenceAfter();
                        const uint32_t cb = h ? c0 : 0u;
                        const uint32_t cnt = h ? p.B - c0 : c0;
                        // child b's position in this half (0xFF: another half)
                        const uint32_t rel = b - cb < cnt ? b - cb : 0xFFu;
                        for (uint32_t c = 0; c < (16u * cnt + 63u) / 64u; c++) {
                            uint32_t r[64];
                            tmemLoad64(tRow + kSlotCols * k + 64u * c, r);
                            tmemWaitTie64(r);
#pragma unroll
                            for (uint32_t kk = 0; kk < 4; kk++)
#pragma unroll
                                for (int i = 0; i < 16; i++) sel[i] = rel == 4u * c + kk ? r[16 * kk + i] : sel[i];
                        }
                        tcFenceBefore();
                        __syncwarp();
                        if (lane == 0) mbarArrive(&S.slotFree[k]);
                    }
                    if (!ok) break;
                    if (row < ti.count) {
                        const uint64_t child = uint64_t(ti.group) * p.B + b; // in-level index at level 2p+1
                        const uint32_t b2 = argminScores(sel, &S.cn[slot][1 + b][0]);
                        emitRow(S, p, smemHist, orig, static_cast<uint32_t>(child * p.B + b2));
                    }
                }
            }
            if (lastOfGroupSmem(S, p, t0, nT, t, ti.group)) {
                __syncwarp();
                if (lane == 0) mbarArrive(&S.bEmpty[slot]);
            }
        }
    }

    tcFenceBefore();
    __syncthreads();
    if (smemHist) {
        for (uint32_t i = threadIdx.x; i < p.nbBins; i += blockDim.x) {
            const uint32_t v = S.hist[i];
            if (v) atomicAdd(&p.binCount[i], v);
        }
    }
    if (warp == 0) {
        tcFenceAfter();
        tmemDealloc(tmem, kTmemCols);
    }
}

// ------------------------------------------------------------------ regroup kernels
// Exclusive scans of the bin histogram: rowOff = scan(count), tileOff = scan(ceil(count/128));
// totals[0] = number of tiles, totals[1] = number of rows.
__global__ void __launch_bounds__(1024) scanBins(const uint32_t* count, uint32_t nb, uint32_t* rowOff,
                                                 uint32_t* tileOff, uint32_t* totals)
{
    __shared__ uint32_t wa[32], wb[32];
    __shared__ uint32_t carryA, carryB;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    if (tid == 0) {
        carryA = 0;
        carryB = 0;
    }
    __syncthreads();
    for (uint32_t base = 0; base < nb; base += 1024) {
        const uint32_t i = base + tid;
        const uint32_t c = i < nb ? count[i] : 0u;
        const uint32_t tc = (c + kTileRows - 1) / kTileRows;
        uint32_t a = c, b = tc;
#pragma unroll
        for (uint32_t off = 1; off < 32; off <<= 1) {
            const uint32_t xa = __shfl_up_sync(0xFFFFFFFFu, a, off);
            const uint32_t xb = __shfl_up_sync(0xFFFFFFFFu, b, off);
            if (lane >= off) {
                a += xa;
                b += xb;
            }
        }
        if (lane == 31) {
            wa[w] = a;
            wb[w] = b;
        }
        __syncthreads();
        if (w == 0) {
            uint32_t va = wa[lane], vb = wb[lane];
#pragma unroll
            for (uint32_t off = 1; off < 32; off <<= 1) {
                const uint32_t xa = __shfl_up_sync(0xFFFFFFFFu, va, off);
                const uint32_t xb = __shfl_up_sync(0xFFFFFFFFu, vb, off);
                if (lane >= off) {
                    va += xa;
                    vb += xb;
                }
            }
            wa[lane] = va; // inclusive over warps
            wb[lane] = vb;
        }
        __syncthreads();
        const uint32_t prevA = (w ? wa[w - 1] : 0u) + carryA;
        const uint32_t prevB = (w ? wb[w - 1] : 0u) + carryB;
        if (i < nb) {
            rowOff[i] = prevA + a - c;
            tileOff[i] = prevB + b - tc;
        }
        __syncthreads();
        if (tid == 0) {
            carryA += wa[31];
            carryB += wb[31];
        }
        __syncthreads();
    }
    if (tid == 0) {
        totals[0] = carryB;
        totals[1] = carryA;
    }
}

// One thread per tile: find its bin (last bin with tileOff <= t) and describe its rows.
__global__ void buildTiles(const uint32_t* count, const uint32_t* rowOff, const uint32_t* tileOff, uint32_t nb,
                           const uint32_t* totals, uint32_t maxTiles, TileInfo* tiles)
{
    const uint32_t nTiles = totals[0];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nTiles && t < maxTiles;
         t += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nb; // first bin with tileOff > t
        while (lo < hi) {
            const uint32_t mid = (lo + hi) / 2;
            if (tileOff[mid] <= t) lo = mid + 1; else hi = mid;
        }
        const uint32_t g = lo - 1;
        const uint32_t k = t - tileOff[g];
        const uint32_t c = count[g] - k * kTileRows;
        tiles[t] = TileInfo{g, rowOff[g] + k * kTileRows, c < kTileRows ? c : kTileRows, 0u};
    }
}

constexpr uint32_t kScatterThreads = 256;

// perm[rowOff[node] + rank] = i for every descriptor i (order inside a bin is unspecified).
// kScatterPerThread rows per thread (8, 16 or 32, chosen by the autotuner).
template <uint32_t kScatterPerThread>
__global__ void __launch_bounds__(kScatterThreads) scatterRows(const uint32_t* nodeNext, uint64_t n, uint32_t nb,
                                                               const uint32_t* rowOff, uint32_t* cursor, uint32_t* perm)
{
    __shared__ uint32_t hist[kSmemHistMax];
    const uint64_t base = uint64_t(blockIdx.x) * kScatterThreads * kScatterPerThread;
    if (nb <= kSmemHistMax) {
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        uint32_t node[kScatterPerThread], rank[kScatterPerThread];
#pragma unroll
        for (uint32_t k = 0; k < kScatterPerThread; k++) {
            const uint64_t i = base + uint64_t(k) * kScatterThreads + threadIdx.x;
            node[k] = i < n ? __ldg(nodeNext + i) : 0xFFFFFFFFu;
            rank[k] = node[k] != 0xFFFFFFFFu ? atomicAdd(&hist[node[k]], 1u) : 0u;
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) {
            const uint32_t c = hist[i];
            hist[i] = c ? atomicAdd(&cursor[i], c) : 0u;
        }
        __syncthreads();
#pragma unroll
        for (uint32_t k = 0; k < kScatterPerThread; k++) {
            const uint64_t i = base + uint64_t(k) * kScatterThreads + threadIdx.x;
            if (node[k] != 0xFFFFFFFFu) perm[rowOff[node[k]] + hist[node[k]] + rank[k]] = static_cast<uint32_t>(i);
        }
    } else {
#pragma unroll
        for (uint32_t k = 0; k < kScatterPerThread; k++) {
            const uint64_t i = base + uint64_t(k) * kScatterThreads + threadIdx.x;
            if (i < n) {
                const uint32_t nd = __ldg(nodeNext + i);
                perm[rowOff[nd] + atomicAdd(&cursor[nd], 1u)] = static_cast<uint32_t>(i);
            }
        }
    }
}

// Regroup of at most kSmemHistMax bins in three kernels, without global atomics: regroupHist
// counts each CTA's contiguous row range per bin (ctaHist[c][b]); regroupScan turns the counts
// into the bins' totals, row and tile offsets and, in place, each (CTA, bin)'s first position;
// regroupScatter hands out those positions again with shared-memory atomics.  Order inside a
// bin is unspecified.
constexpr uint32_t kRegroupThreads = 1024;

__device__ __forceinline__ void regroupRange(uint64_t n, uint64_t per, uint64_t& beg, uint64_t& end)
{
    beg = uint64_t(blockIdx.x) * per;
    end = beg + per < n ? beg + per : n;
    if (beg > end) beg = end;
}

// f(node, row) for every row of this CTA's range; four rows per 16-byte load, four loads in flight.
template <typename F>
__device__ __forceinline__ void forEachRow(const uint32_t* nodeNext, uint64_t beg, uint64_t end, F f)
{
    // per is a multiple of 16 rows, so beg is 64-byte aligned
    const uint64_t nVec = (end - beg) / 4;
    const uint4* v4 = reinterpret_cast<const uint4*>(nodeNext + beg);
    uint64_t j = threadIdx.x;
    for (; j + 3 * kRegroupThreads < nVec; j += 4 * kRegroupThreads) {
        uint4 v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) v[u] = __ldg(v4 + j + u * kRegroupThreads);
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t r = beg + 4 * (j + u * kRegroupThreads);
            f(v[u].x, r);
            f(v[u].y, r + 1);
            f(v[u].z, r + 2);
            f(v[u].w, r + 3);
        }
    }
    for (; j < nVec; j += kRegroupThreads) {
        const uint4 v = __ldg(v4 + j);
        const uint64_t r = beg + 4 * j;
        f(v.x, r);
        f(v.y, r + 1);
        f(v.z, r + 2);
        f(v.w, r + 3);
    }
    for (uint64_t r = beg + 4 * nVec + threadIdx.x; r < end; r += kRegroupThreads) f(__ldg(nodeNext + r), r);
}

__global__ void __launch_bounds__(kRegroupThreads) regroupHist(const uint32_t* nodeNext, uint64_t n, uint64_t per,
                                                               uint32_t nb, uint32_t* ctaHist)
{
    __shared__ uint32_t hist[kSmemHistMax];
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    uint64_t beg, end;
    regroupRange(n, per, beg, end);
    forEachRow(nodeNext, beg, end, [&](uint32_t node, uint64_t) { atomicAdd(&hist[node], 1u); });
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) ctaHist[uint64_t(blockIdx.x) * nb + i] = hist[i];
}

// One CTA of 1024 threads: thread (k, b) owns bin b's CTAs [k * len, (k + 1) * len).
__global__ void __launch_bounds__(1024) regroupScan(uint32_t* ctaHist, uint32_t nCta, uint32_t nb, uint32_t* count,
                                                    uint32_t* rowOff, uint32_t* tileOff, uint32_t* totals)
{
    __shared__ uint32_t part[1024];
    __shared__ uint32_t wa[32], wb[32];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    const uint32_t chunks = 1024 / nb;                    // >= 1 (nb <= 1024)
    const uint32_t len = (nCta + chunks - 1) / chunks;
    const uint32_t b = tid % nb, k = tid / nb;
    const bool active = k < chunks;
    const uint32_t c0 = active ? k * len : nCta;
    const uint32_t c1 = active ? min(nCta, c0 + len) : nCta;
    // eight loads in flight per step (the loop is bound by load latency)
    uint32_t sum = 0;
    for (uint32_t c = c0; c < c1; c += 8) {
        uint32_t v[8];
#pragma unroll
        for (uint32_t u = 0; u < 8; u++) v[u] = c + u < c1 ? ctaHist[uint64_t(c + u) * nb + b] : 0u;
#pragma unroll
        for (uint32_t u = 0; u < 8; u++) sum += v[u];
    }
    part[tid] = sum;
    __syncthreads();
    // bin totals and the chunk's prefix inside its bin
    uint32_t before = 0, total = 0;
    if (active) {
        for (uint32_t kk = 0; kk < chunks; kk++) {
            const uint32_t v = part[kk * nb + b];
            if (kk < k) before += v;
            total += v;
        }
    }
    // exclusive scans over bins of total and ceil(total / 128) (threads k == 0 hold the bins)
    const bool owner = active && k == 0;
    const uint32_t ca = owner ? total : 0u, cb = owner ? (total + kTileRows - 1) / kTileRows : 0u;
    uint32_t a = ca, t = cb;
#pragma unroll
    for (uint32_t off = 1; off < 32; off <<= 1) {
        const uint32_t xa = __shfl_up_sync(0xFFFFFFFFu, a, off);
        const uint32_t xb = __shfl_up_sync(0xFFFFFFFFu, t, off);
        if (lane >= off) {
            a += xa;
            t += xb;
        }
    }
    if (lane == 31) {
        wa[w] = a;
        wb[w] = t;
    }
    __syncthreads();
    if (w == 0) {
        uint32_t va = wa[lane], vb = wb[lane];
#pragma unroll
        for (uint32_t off = 1; off < 32; off <<= 1) {
            const uint32_t xa = __shfl_up_sync(0xFFFFFFFFu, va, off);
            const uint32_t xb = __shfl_up_sync(0xFFFFFFFFu, vb, off);
            if (lane >= off) {
                va += xa;
                vb += xb;
            }
        }
        wa[lane] = va;
        wb[lane] = vb;
    }
    __syncthreads();
    const uint32_t exA = (w ? wa[w - 1] : 0u) + a - ca;
    const uint32_t exB = (w ? wb[w - 1] : 0u) + t - cb;
    if (owner) {
        count[b] = total;
        rowOff[b] = exA;
        tileOff[b] = exB;
        part[b] = exA; // the bin's first row, for the other chunks (read after the barrier)
    }
    if (tid == 1023) {
        totals[0] = wb[31];
        totals[1] = wa[31];
    }
    __syncthreads();
    if (active) {
        uint32_t run = part[b] + before;
        for (uint32_t c = c0; c < c1; c += 8) {
            uint32_t v[8];
#pragma unroll
            for (uint32_t u = 0; u < 8; u++) v[u] = c + u < c1 ? ctaHist[uint64_t(c + u) * nb + b] : 0u;
#pragma unroll
            for (uint32_t u = 0; u < 8; u++) {
                if (c + u < c1) ctaHist[uint64_t(c + u) * nb + b] = run;
                run += v[u];
            }
        }
    }
}

// Chunks of kScatterChunk rows are grouped by bin in shared memory first, so each bin's rows of a
// chunk leave as one contiguous run of the permutation (whole sectors) rather than as scattered
// 4-byte stores.
constexpr uint32_t kScatterChunk = 8192;
constexpr uint32_t kScatterPerThread = kScatterChunk / kRegroupThreads;
constexpr size_t kScatterSmemBytes = size_t(kScatterChunk) * 6 + 2 * kSmemHistMax * 4;

__global__ void __launch_bounds__(kRegroupThreads) regroupScatter(const uint32_t* nodeNext, uint64_t n, uint64_t per,
                                                                  uint32_t nb, const uint32_t* ctaOff, uint32_t* perm)
{
    extern __shared__ uint32_t smemScatter[];
    uint32_t* next = smemScatter;                  // [nb] position of this CTA's next row per bin
    uint32_t* cnt = next + kSmemHistMax;           // [nb] rows of the chunk per bin, then offsets
    uint32_t* stage = cnt + kSmemHistMax;          // [kScatterChunk] row ids grouped by bin
    uint16_t* stageBin = reinterpret_cast<uint16_t*>(stage + kScatterChunk);
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) next[i] = ctaOff[uint64_t(blockIdx.x) * nb + i];
    uint64_t beg, end;
    regroupRange(n, per, beg, end);
    for (uint64_t c0 = beg; c0 < end; c0 += kScatterChunk) {
        const uint32_t rows = static_cast<uint32_t>(end - c0 < kScatterChunk ? end - c0 : kScatterChunk);
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) cnt[i] = 0;
        __syncthreads();
        uint32_t node[kScatterPerThread], rank[kScatterPerThread];
#pragma unroll
        for (uint32_t k = 0; k < kScatterPerThread; k++) {
            const uint32_t j = k * kRegroupThreads + threadIdx.x;
            node[k] = j < rows ? __ldg(nodeNext + c0 + j) : 0u;
        }
#pragma unroll
        for (uint32_t k = 0; k < kScatterPerThread; k++)
            if (k * kRegroupThreads + threadIdx.x < rows) rank[k] = atomicAdd(&cnt[node[k]], 1u);
        __syncthreads();
        if (threadIdx.x < 32) {
            // exclusive scan of the chunk's bin counts in place (lane l: bins 32 l .. 32 l + 31)
            const uint32_t lane = threadIdx.x;
            uint32_t sum = 0;
            for (uint32_t i = 32 * lane; i < 32 * lane + 32 && i < nb; i++) sum += cnt[i];
            uint32_t incl = sum;
#pragma unroll
            for (uint32_t off = 1; off < 32; off <<= 1) {
                const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
                if (lane >= off) incl += v;
            }
            uint32_t run = incl - sum;
            for (uint32_t i = 32 * lane; i < 32 * lane + 32 && i < nb; i++) {
                const uint32_t c = cnt[i];
                cnt[i] = run;
                run += c;
            }
        }
        __syncthreads();
#pragma unroll
        for (uint32_t k = 0; k < kScatterPerThread; k++) {
            const uint32_t j = k * kRegroupThreads + threadIdx.x;
            if (j < rows) {
                const uint32_t at = cnt[node[k]] + rank[k];
                stage[at] = static_cast<uint32_t>(c0 + j);
                stageBin[at] = static_cast<uint16_t>(node[k]);
            }
        }
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < rows; j += blockDim.x) {
            const uint32_t bn = stageBin[j];
            perm[next[bn] + (j - cnt[bn])] = stage[j];
        }
        __syncthreads();
        // the chunk's count of bin b is the distance to the next bin's offset
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) next[i] += (i + 1 < nb ? cnt[i + 1] : rows) - cnt[i];
        __syncthreads();
    }
}

// ------------------------------------------------------------------ plain FP32 SIMT kernel
// One thread per descriptor.  The block's 128 descriptor rows are staged once in shared memory
// (coalesced 16-byte loads; rows padded to 144 bytes so that the eight 16-byte reads of a
// quarter warp fall in distinct banks).  Per level the thread walks its row in 16-dimension
// chunks: the chunk is converted to fp32 once and multiplied into 16 fp32 accumulators, one per
// center, whose bytes are read as 16-byte vectors from the tree (L1/L2) and converted to fp32
// on the fly.  Every partial sum is an integer below 2^24, so the fp32 dot products -- and
// |c|^2 - 2 x.c -- are exact and the argmin (lowest index on ties) equals the reference's.
constexpr uint32_t kSimtThreads = 128;
constexpr uint32_t kSimtRowStride = kDims + 16;

__device__ __forceinline__ float byteToFloat(uint32_t word, uint32_t k)
{
    // 0x4B0000bb is the float 2^23 + bb; subtracting 2^23 leaves bb exactly.
    return __int_as_float(static_cast<int>(__byte_perm(word, 0x4B000000u, 0x7540u | k))) - 8388608.0f;
}

__global__ void __launch_bounds__(kSimtThreads, 8) lookupSimtF32(const uint8_t* __restrict__ centers,
                                                              const int32_t* __restrict__ cnorm, uint32_t B,
                                                              uint32_t L, const uint8_t* __restrict__ desc,
                                                              uint64_t n, uint32_t* __restrict__ out)
{
    __shared__ __align__(16) uint8_t xs[kSimtThreads * kSimtRowStride];
    const uint64_t base = uint64_t(blockIdx.x) * kSimtThreads;
#pragma unroll
    for (uint32_t k = 0; k < 8; k++) {
        const uint32_t i = k * kSimtThreads + threadIdx.x; // 16-byte chunk i % 8 of row i / 8
        const uint32_t r = i / 8, c = i % 8;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (base + r < n) v = __ldg(reinterpret_cast<const uint4*>(desc + (base + r) * kDims) + c);
        *reinterpret_cast<uint4*>(xs + r * kSimtRowStride + c * 16) = v;
    }
    __syncthreads();
    const uint8_t* x = xs + threadIdx.x * kSimtRowStride;
    uint64_t idx = 0, lb = 0;
    for (uint32_t level = 0; level < L; level++) {
        const uint64_t node = lb + idx;
        const uint4* c4 = reinterpret_cast<const uint4*>(centers + node * kMaxBranch * kDims);
        float acc[kMaxBranch];
#pragma unroll
        for (uint32_t b = 0; b < kMaxBranch; b++) acc[b] = 0.f;
#pragma unroll 1
        for (uint32_t chunk = 0; chunk < 8; chunk++) {
            const uint4 xv = *reinterpret_cast<const uint4*>(x + chunk * 16);
            const uint32_t xw[4] = {xv.x, xv.y, xv.z, xv.w};
            float xf[16];
#pragma unroll
            for (uint32_t q = 0; q < 4; q++)
#pragma unroll
                for (uint32_t k = 0; k < 4; k++) xf[4 * q + k] = byteToFloat(xw[q], k);
#pragma unroll
            for (uint32_t b = 0; b < kMaxBranch; b++) {
                if (b < B) {
                    const uint4 cv = __ldg(c4 + b * 8 + chunk);
                    const uint32_t cw[4] = {cv.x, cv.y, cv.z, cv.w};
#pragma unroll
                    for (uint32_t q = 0; q < 4; q++)
#pragma unroll
                        for (uint32_t k = 0; k < 4; k++) acc[b] = fmaf(xf[4 * q + k], byteToFloat(cw[q], k), acc[b]);
                }
            }
        }
        const int32_t* cn = cnorm + node * kMaxBranch;
        float best = static_cast<float>(__ldg(cn)) - 2.f * acc[0];
        uint32_t bi = 0;
#pragma unroll
        for (uint32_t b = 1; b < kMaxBranch; b++) {
            if (b < B) {
                const float s = static_cast<float>(__ldg(cn + b)) - 2.f * acc[b];
                if (s < best) {
                    best = s;
                    bi = b;
                }
            }
        }
        idx = idx * B + bi;
        lb = lb * B + 1;
    }
    if (base + threadIdx.x < n) out[base + threadIdx.x] = static_cast<uint32_t>(idx);
}

// ------------------------------------------------------------------ host side
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encodeTiledFn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<EncodeTiledFn>(p);
        }
    });
    if (fn == nullptr) throw Error(kCudaError, "cuTensorMapEncodeTiled is unavailable");
    return fn;
}

CUtensorMap makeRowMap(const uint8_t* desc, uint64_t n, uint32_t boxRows)
{
    CUtensorMap m{};
    const cuuint64_t dims[2] = {kDims, n};
    const cuuint64_t strides[1] = {kDims};
    const cuuint32_t box[2] = {kDims, boxRows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encodeTiledFn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(desc), dims, strides,
                                       box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(kCudaError, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
    return m;
}

uint32_t maxBinsFor(uint32_t B, uint32_t L)
{
    uint64_t m = 1;
    const uint32_t passes = (L + 1) / 2;
    for (uint32_t p = 0; p + 1 < passes; p++) m = std::max<uint64_t>(m, ipow(B, 2 * p + 2));
    return static_cast<uint32_t>(m);
}

// Words of the per-CTA histograms: regroups of at most kSmemHistMax bins use them.
uint64_t ctaHistWords(uint32_t B, uint32_t L)
{
    uint64_t m = 0;
    const uint32_t passes = (L + 1) / 2;
    for (uint32_t p = 0; p + 1 < passes; p++) {
        const uint64_t nb = ipow(B, 2 * p + 2);
        if (nb <= kSmemHistMax) m = std::max<uint64_t>(m, nb);
    }
    return m * kRegroupCtas;
}

} // namespace

size_t lookupScratchBytes(uint32_t B, uint32_t L, uint64_t n)
{
    if (L <= 2) return 256; // single pass: no regroup (only the error record)
    const uint64_t bins = maxBinsFor(B, L);
    const uint64_t tiles = n / kTileRows + bins + 1;
    auto a = [](uint64_t b) { return (b + 255) / 256 * 256; };
    return a(sizeof(DeviceErrors)) + 2 * a(n * 4) + a((4 * bins + 4) * 4) + a(tiles * sizeof(TileInfo)) +
           a(ctaHistWords(B, L) * 4);
}

LookupScratch carveLookupScratch(void* base, uint32_t B, uint32_t L, uint64_t n)
{
    LookupScratch s{};
    auto a = [](uint64_t b) { return (b + 255) / 256 * 256; };
    uint8_t* p = static_cast<uint8_t*>(base);
    s.err = reinterpret_cast<DeviceErrors*>(p);
    p += a(sizeof(DeviceErrors));
    if (L <= 2) return s;
    const uint64_t bins = maxBinsFor(B, L);
    s.nodeNext = reinterpret_cast<uint32_t*>(p);
    p += a(n * 4);
    s.perm = reinterpret_cast<uint32_t*>(p);
    p += a(n * 4);
    s.bins = reinterpret_cast<uint32_t*>(p);
    p += a((4 * bins + 4) * 4);
    s.tiles = p;
    p += a((n / kTileRows + bins + 1) * sizeof(TileInfo));
    s.ctaHist = reinterpret_cast<uint32_t*>(p);
    return s;
}

uint32_t launchLookup(const DeviceTree& tree, const uint8_t* desc, uint64_t n, uint32_t* leaf, LookupAlgo algo,
                      const LookupScratch& scratch, cudaStream_t stream)
{
    if (n == 0) return 0;
    if (algo == kLookupSimtF32) {
        const uint64_t blocks = (n + kSimtThreads - 1) / kSimtThreads;
        ScopedKernelTimer timer(kTimedLookupSimt, stream);
        lookupSimtF32<<<static_cast<uint32_t>(blocks), kSimtThreads, 0, stream>>>(tree.centers, tree.cnorm, tree.B, tree.L, desc,
                                                                         n, leaf);
        RBW_CUDA(cudaGetLastError());
        return 1;
    }
    const bool warpNode = algo == kLookupTensorU8WarpNode;
    const bool ring = algo == kLookupTensorU8Ring;
    static std::atomic<uint64_t> attrSet{0}, attrSetW{0}, attrSetR{0}, attrSetS{0};
    setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(regroupScatter), static_cast<int>(kScatterSmemBytes),
                                   attrSetS);
    if (ring) {
        setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(lookupPassRing),
                                       static_cast<int>(kTcSmemBytes), attrSetR);
    } else if (warpNode) {
        setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(lookupPassTc<true>),
                                       static_cast<int>(kTcSmemBytes), attrSetW);
    } else {
        setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(lookupPassTc<false>),
                                       static_cast<int>(kTcSmemBytes), attrSet);
    }
    const CUtensorMap tmapTile = makeRowMap(desc, n, kTileRows);
    const uint32_t B = tree.B, L = tree.L;
    const uint32_t passes = (L + 1) / 2;
    const uint32_t grid = static_cast<uint32_t>(currentSmCount());
    const uint64_t bins = L > 2 ? maxBinsFor(B, L) : 0;
    uint32_t* count = scratch.bins;
    uint32_t* rowOff = count ? count + bins : nullptr;
    uint32_t* tileOff = count ? rowOff + bins : nullptr;
    uint32_t* cursor = count ? tileOff + bins : nullptr;
    uint32_t* totals = count ? cursor + bins : nullptr;
    TileInfo* tiles = static_cast<TileInfo*>(scratch.tiles);
    const uint32_t maxTiles = static_cast<uint32_t>(n / kTileRows + bins + 1);
    uint32_t kernels = 0;
    for (uint32_t pass = 0; pass < passes; pass++) {
        PassParams p{};
        p.desc = desc;
        p.centersSw = tree.centersSw;
        p.cnorm = tree.cnorm;
        p.B = B;
        p.twoLevels = (2 * pass + 1 < L) ? 1u : 0u;
        p.lbA = levelBeg(B, 2 * pass);
        p.lbB = levelBeg(B, 2 * pass + 1);
        p.nRows = n;
        p.isFinal = pass + 1 == passes;
        p.err = scratch.err;
        if (pass > 0) {
            p.perm = scratch.perm;
            p.tiles = tiles;
            p.nTilesDev = totals;
        }
        uint32_t nbBins = 0;
        // regroups of at most kSmemHistMax bins count per CTA in regroupHist; larger ones in the pass
        bool ctaRegroup = false;
        if (p.isFinal) {
            p.out = leaf;
        } else {
            nbBins = static_cast<uint32_t>(ipow(B, 2 * pass + 2));
            ctaRegroup = nbBins <= kSmemHistMax && scratch.ctaHist != nullptr;
            p.nodeNext = scratch.nodeNext;
            p.binCount = ctaRegroup ? nullptr : count;
            p.nbBins = nbBins;
            if (!ctaRegroup) RBW_CUDA(cudaMemsetAsync(count, 0, sizeof(uint32_t) * nbBins, stream));
        }
        {
            ScopedKernelTimer timer(kTimedLookupPass, stream);
            if (ring) {
                lookupPassRing<<<grid, kRingThreads, kTcSmemBytes, stream>>>(tmapTile, p);
            } else if (warpNode) {
                lookupPassTc<true><<<grid, kTcThreads, kTcSmemBytes, stream>>>(tmapTile, p);
            } else {
                lookupPassTc<false><<<grid, kTcThreads, kTcSmemBytes, stream>>>(tmapTile, p);
            }
            RBW_CUDA(cudaGetLastError());
        }
        kernels++;
        if (!p.isFinal) {
            ScopedKernelTimer timer(kTimedRegroup, stream);
            const uint32_t tileBlocks = std::min<uint32_t>((maxTiles + 255) / 256, 4096);
            if (ctaRegroup) {
                const uint64_t per = ((n + kRegroupCtas - 1) / kRegroupCtas + 15) / 16 * 16;
                regroupHist<<<kRegroupCtas, kRegroupThreads, 0, stream>>>(scratch.nodeNext, n, per, nbBins,
                                                                         scratch.ctaHist);
                regroupScan<<<1, 1024, 0, stream>>>(scratch.ctaHist, kRegroupCtas, nbBins, count, rowOff, tileOff,
                                                    totals);
                buildTiles<<<tileBlocks, 256, 0, stream>>>(count, rowOff, tileOff, nbBins, totals, maxTiles, tiles);
                regroupScatter<<<kRegroupCtas, kRegroupThreads, kScatterSmemBytes, stream>>>(
                    scratch.nodeNext, n, per, nbBins, scratch.ctaHist, scratch.perm);
                RBW_CUDA(cudaGetLastError());
                kernels += 4;
                continue;
            }
            scanBins<<<1, 1024, 0, stream>>>(count, nbBins, rowOff, tileOff, totals);
            RBW_CUDA(cudaGetLastError());
            buildTiles<<<tileBlocks, 256, 0, stream>>>(count, rowOff, tileOff, nbBins, totals, maxTiles, tiles);
            RBW_CUDA(cudaGetLastError());
            RBW_CUDA(cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * nbBins, stream));
            const uint32_t rows = tunedValue(kTuneScatterRows, B, L, n);
            const uint64_t per = uint64_t(kScatterThreads) * rows;
            const uint32_t sBlocks = static_cast<uint32_t>((n + per - 1) / per);
            if (rows == 8) {
                scatterRows<8><<<sBlocks, kScatterThreads, 0, stream>>>(scratch.nodeNext, n, nbBins, rowOff, cursor,
                                                                          scratch.perm);
            } else if (rows == 32) {
                scatterRows<32><<<sBlocks, kScatterThreads, 0, stream>>>(scratch.nodeNext, n, nbBins, rowOff, cursor,
                                                                           scratch.perm);
            } else {
                scatterRows<16><<<sBlocks, kScatterThreads, 0, stream>>>(scratch.nodeNext, n, nbBins, rowOff, cursor,
                                                                           scratch.perm);
            }
            RBW_CUDA(cudaGetLastError());
            kernels += 3;
        }
    }
    return kernels;
}

} // namespace rbw
