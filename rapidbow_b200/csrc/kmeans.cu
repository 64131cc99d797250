// Hierarchical k-means kernels.  Distances are exact integers: score_b = |c_b|^2 - 2 x.c_b with
// x.c_b from the tensor core (tcgen05.mma.kind::i8, u8 x u8 -> s32) in the assign step and from
// dp4a in k-means++, argmin with the lowest index on ties (kmeans.cu:131-135).
// Center sums are exact (u32 in shared memory, u64 in global memory).
#include "kmeans.cuh"
#include "timing.h"
#include "tuning.h"

#include <algorithm>

namespace rbw {
namespace {

constexpr uint32_t kScanBlock = 1024;
constexpr uint32_t kScanPerThread = 4;
constexpr uint32_t kScanTile = kScanBlock * kScanPerThread;

__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* warpSums, uint32_t& total)
{
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (uint32_t off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warpSums[w] = x;
    __syncthreads();
    if (w == 0) {
        const uint32_t nw = blockDim.x / 32;
        uint32_t s = lane < nw ? warpSums[lane] : 0u;
#pragma unroll
        for (uint32_t off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, off);
            if (lane >= off) s += y;
        }
        warpSums[lane] = s;
    }
    __syncthreads();
    total = warpSums[blockDim.x / 32 - 1];
    const uint32_t r = (w ? warpSums[w - 1] : 0u) + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanBlock) scanBlockSums(const uint32_t* in, uint64_t n, uint32_t* blockSums)
{
    __shared__ uint32_t ws[32];
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile + threadIdx.x * kScanPerThread;
    uint32_t s = 0;
#pragma unroll
    for (uint32_t k = 0; k < kScanPerThread; k++)
        if (base + k < n) s += in[base + k];
    uint32_t total;
    blockExclusiveScan(s, ws, total);
    if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) scanSingle(uint32_t* data, uint32_t n)
{
    __shared__ uint32_t ws[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += kScanBlock) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n ? data[i] : 0u;
        uint32_t total;
        const uint32_t e = blockExclusiveScan(v, ws, total);
        if (i < n) data[i] = e + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanBlock) scanApply(const uint32_t* in, uint64_t n, const uint32_t* blockOff,
                                                        uint32_t* out)
{
    __shared__ uint32_t ws[32];
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile + threadIdx.x * kScanPerThread;
    uint32_t v[kScanPerThread];
    uint32_t s = 0;
#pragma unroll
    for (uint32_t k = 0; k < kScanPerThread; k++) {
        v[k] = base + k < n ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t e = blockExclusiveScan(s, ws, total) + blockOff[blockIdx.x];
#pragma unroll
    for (uint32_t k = 0; k < kScanPerThread; k++) {
        if (base + k < n) out[base + k] = e;
        e += v[k];
    }
}

__global__ void ceilDivKernel(const uint32_t* cnt, uint32_t n, uint32_t d, uint32_t* out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (cnt[i] + d - 1) / d;
}

__global__ void tilesTotal(const uint32_t* cnt, const uint32_t* tileOff, uint32_t n, uint32_t d, uint32_t* totals)
{
    if (n == 0) {
        totals[0] = 0;
        return;
    }
    totals[0] = tileOff[n - 1] + (cnt[n - 1] + d - 1) / d;
}

__global__ void fillNodeTiles(const uint32_t* cnt, const uint32_t* off, const uint32_t* tileOff, uint32_t nbNodes,
                              uint32_t d, const uint32_t* totals, uint32_t maxTiles, NodeTile* tiles)
{
    const uint32_t nTiles = totals[0];
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nTiles && t < maxTiles;
         t += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nbNodes;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) / 2;
            if (tileOff[mid] <= t) lo = mid + 1; else hi = mid;
        }
        const uint32_t g = lo - 1;
        const uint32_t k = t - tileOff[g];
        const uint32_t c = cnt[g] - k * d;
        tiles[t] = NodeTile{g, off[g] + k * d, c < d ? c : d, tileOff[g]};
    }
}

// ------------------------------------------------------------------ centers
__global__ void initCentersKernel(KMeansLevel lv, const uint32_t* pos, uint64_t nbDescTotal, int posIsDesc)
{
    // thread per (node, slot, 16-byte chunk)
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t total = uint64_t(lv.nbNodes) * kMaxBranch * 8;
    if (i >= total) return;
    const uint32_t chunk = i % 8;
    const uint32_t b = (i / 8) % kMaxBranch;
    const uint32_t g = static_cast<uint32_t>(i / (8 * kMaxBranch));
    uint4 v = make_uint4(0, 0, 0, 0);
    if (b < lv.B) {
        const uint32_t p = pos[uint64_t(g) * lv.B + b];
        const uint64_t at = posIsDesc ? uint64_t(p) : uint64_t(lv.nodeOff[g]) + p;
        if (p != kInvalidIdx && at < (posIsDesc ? nbDescTotal : lv.nbMembers)) {
            const uint32_t d = posIsDesc ? p : lv.members[at];
            v = reinterpret_cast<const uint4*>(lv.desc + uint64_t(d) * kDims)[chunk];
        } else {
            v = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        }
    }
    reinterpret_cast<uint4*>(lv.centers + (uint64_t(g) * kMaxBranch + b) * kDims)[chunk] = v;
}

__global__ void centerNormsKernel(KMeansLevel lv)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= uint64_t(lv.nbNodes) * kMaxBranch) return;
    const uint32_t b = i % kMaxBranch;
    if (b >= lv.B) {
        lv.cnorm[i] = kPadNorm;
        return;
    }
    const uint4* c = reinterpret_cast<const uint4*>(lv.centers + i * kDims);
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint4 v = c[k];
        acc = __dp4a(v.x, v.x, acc);
        acc = __dp4a(v.y, v.y, acc);
        acc = __dp4a(v.z, v.z, acc);
        acc = __dp4a(v.w, v.w, acc);
    }
    lv.cnorm[i] = static_cast<int32_t>(acc);
}

// ------------------------------------------------------------------ k-means++ init
// SplitMix64 (Steele, Lea, Flood 2014): the output for state z; the generator adds
// kSplitMixGamma to the state before each output, so draw i (from 0) of a stream started at s
// is splitMixOut(s + (i + 1) * kSplitMixGamma).
constexpr uint64_t kSplitMixGamma = 0x9E3779B97F4A7C15ull;
__device__ __forceinline__ uint64_t splitMixOut(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t splitmix64(uint64_t& s)
{
    s += kSplitMixGamma;
    return splitMixOut(s);
}

constexpr uint32_t kPPSample = 256;
constexpr uint32_t kPPWarps = kPPSample / 32;
constexpr uint32_t kPPCtasPerSm = 6; // by shared memory: 32 KB of candidate rows per CTA

// One CTA (256 threads) per node.  Same specification as the oracle's orc_kmeanspp_init:
// SplitMix64 stream seeded by (seed, level, node); Floyd sampling of min(n, 256) member
// positions (sorted); first center uniform; then D^2 sampling with exact integer weights.
// Floyd's draws do not depend on the set, so thread m makes draw m, t_m = out_m % (j_m + 1) with
// j_m = n - 256 + m, directly from the counter-based stream.  Step m inserts j_m when t_m is
// already in the set, else t_m; with base = n - 256:
//   - t_m < base: t_m is in the set iff an earlier draw equals it (values below base enter only
//     as themselves, and the first equal draw did enter);
//   - t_m = base + m: not yet in the set (every earlier value is below j_m);
//   - t_m = j_r, r < m: in the set iff step r inserted j_r (found_r) or a draw t_q, r <= q < m,
//     equals it;
// so found_m = local_m || found_r along links m -> r < m, an OR over a chain of at most 256
// steps, resolved by eight rounds of pointer jumping.  The distinct positions are then sorted by
// rank (each thread counts the smaller ones).  The candidate rows sit in shared memory and thread
// i holds candidate i's D^2 weight; each pick's prefix sums are warp scans plus one pass over the
// eight warp totals, and every thread draws the same random numbers, so a pick costs two
// barriers.  Registers stay low enough for six CTAs per SM (deep levels have 10^5 nodes).
__global__ void __launch_bounds__(kPPSample, kPPCtasPerSm) kmeansPPKernel(KMeansLevel lv, uint64_t seed,
                                                                          uint32_t level, uint32_t* nValidOut)
{
    // candidate rows, chunk c of row i at [i][c ^ (i & 7)] (a quarter-warp reading its own rows
    // hits 32 different banks)
    __shared__ uint4 rowS[kPPSample][kDims / 16];
    __shared__ uint32_t pos[kPPSample];
    __shared__ uint32_t cand[kPPSample];
    __shared__ uint32_t draw[kPPSample];
    __shared__ uint32_t link[kPPSample];
    __shared__ uint8_t found[kPPSample];
    __shared__ unsigned long long warpSum[kPPWarps];
    __shared__ uint32_t chosen[kMaxBranch];
    const uint32_t g = blockIdx.x;
    const uint32_t n = lv.nodeCnt[g];
    const uint32_t tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
    const uint32_t S = n < kPPSample ? n : kPPSample;
    if (n == 0) {
        if (tid == 0) nValidOut[g] = 0;
        for (uint32_t i = tid; i < kMaxBranch * 8; i += blockDim.x) {
            reinterpret_cast<uint4*>(lv.centers + uint64_t(g) * kMaxBranch * kDims)[i] =
                make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        }
        return;
    }
    uint64_t s = seed ^ (uint64_t(level) * 0x9E3779B97F4A7C15ull) ^ (uint64_t(g) * 0xD1B54A32D192ED03ull);
    if (n > kPPSample) {
        constexpr uint32_t kNone = 0xFFFFFFFFu;
        const uint32_t base = n - kPPSample;
        const uint32_t t = static_cast<uint32_t>(splitMixOut(s + uint64_t(tid + 1) * kSplitMixGamma) %
                                                 (uint64_t(base) + tid + 1));
        draw[tid] = t;
        __syncthreads();
        bool f = false;
        uint32_t lk = kNone, q0 = 0;
        if (t >= base) {
            const uint32_t r = t - base;
            q0 = r < tid ? r : tid; // r == tid: nothing to compare, no link
            if (r < tid) lk = r;
        }
        for (uint32_t q = q0; q < tid; q++) f |= draw[q] == t;
        found[tid] = f ? 1 : 0;
        link[tid] = lk;
        __syncthreads();
#pragma unroll 1
        for (uint32_t round = 0; round < 8; round++) {
            bool nf = f;
            uint32_t nl = lk;
            if (lk != kNone) {
                nf = f || found[lk] != 0;
                nl = link[lk];
            }
            __syncthreads();
            f = nf;
            lk = nl;
            found[tid] = f ? 1 : 0;
            link[tid] = lk;
            __syncthreads();
        }
        pos[tid] = f ? base + tid : t;
        s += uint64_t(kPPSample) * kSplitMixGamma; // the stream after the 256 draws
        __syncthreads();
        // ascending order: the positions are distinct, so each one's rank is its slot
        const uint32_t v = pos[tid];
        uint32_t rk = 0;
        for (uint32_t q = 0; q < kPPSample; q++) rk += pos[q] < v ? 1u : 0u;
        cand[rk] = lv.members[lv.nodeOff[g] + v];
    } else if (tid < S) {
        cand[tid] = lv.members[lv.nodeOff[g] + tid];
    }
    __syncthreads();
    const bool mine = tid < S;
    // eight threads per row, 32 rows per round
#pragma unroll
    for (uint32_t k = 0; k < kPPSample / 32; k++) {
        const uint32_t r = 32u * k + tid / 8, c = tid % 8;
        if (r < S) rowS[r][c ^ (r & 7u)] = reinterpret_cast<const uint4*>(lv.desc + uint64_t(cand[r]) * kDims)[c];
    }
    // the squared distance of this thread's row to row p
    auto distTo = [&](uint32_t p) -> unsigned long long {
        uint32_t acc = 0;
#pragma unroll
        for (uint32_t c = 0; c < kDims / 16; c++) {
            const uint4 x = rowS[tid][c ^ (tid & 7u)], y = rowS[p][c ^ (p & 7u)];
            const uint32_t d0 = __vabsdiffu4(x.x, y.x), d1 = __vabsdiffu4(x.y, y.y);
            const uint32_t d2v = __vabsdiffu4(x.z, y.z), d3 = __vabsdiffu4(x.w, y.w);
            acc = __dp4a(d0, d0, acc);
            acc = __dp4a(d1, d1, acc);
            acc = __dp4a(d2v, d2v, acc);
            acc = __dp4a(d3, d3, acc);
        }
        return acc;
    };
    const uint32_t pick = static_cast<uint32_t>(splitmix64(s) % S);
    if (tid == 0) chosen[0] = pick;
    __syncthreads();
    unsigned long long d2 = mine ? distTo(pick) : 0ull;
    uint32_t nv = 1;
    for (uint32_t k = 1; k < lv.B; k++) {
        // inclusive prefix of d2 over the candidates: warp scan, then the earlier warps' totals
        unsigned long long incl = d2;
#pragma unroll
        for (uint32_t off = 1; off < 32; off <<= 1) {
            const unsigned long long v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
            if (lane >= off) incl += v;
        }
        if (lane == 31) warpSum[warp] = incl;
        __syncthreads();
        unsigned long long before = 0, total = 0;
#pragma unroll
        for (uint32_t w = 0; w < kPPWarps; w++) {
            const unsigned long long v = warpSum[w];
            before += w < warp ? v : 0ull;
            total += v;
        }
        if (total == 0) break; // uniform across the CTA
        incl += before;
        const unsigned long long t = splitmix64(s) % total;
        // smallest i with prefix[i] > t: exactly one candidate has prefix > t >= prefix - d2
        const bool hit = mine && incl > t && incl - d2 <= t;
        if (hit) chosen[k] = tid;
        nv = k + 1;
        __syncthreads();
        if (mine) {
            const unsigned long long d = distTo(chosen[k]);
            if (d < d2) d2 = d;
        }
        __syncthreads(); // warpSum is rewritten by the next pick
    }
    if (tid == 0) nValidOut[g] = nv;
    for (uint32_t i = tid; i < kMaxBranch * 8; i += blockDim.x) {
        const uint32_t b = i / 8, chunk = i % 8;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (b < lv.B) {
            const uint32_t c = cand[chosen[b < nv ? b : nv - 1]];
            v = reinterpret_cast<const uint4*>(lv.desc + uint64_t(c) * kDims)[chunk];
        }
        reinterpret_cast<uint4*>(lv.centers + (uint64_t(g) * kMaxBranch + b) * kDims)[chunk] = v;
    }
}

// ------------------------------------------------------------------ assign
// One step handles one 128-member tile of one node (the reference's DescTile groups,
// kmeans.cu:62-211, on the tensor core):
//   1. the members' rows are gathered into shared memory in the 128-byte swizzled K-major layout
//      (eight threads per row), next to the node's 16 centers in the same layout;
//   2. one thread issues four tcgen05.mma.kind::i8 (M = 128 members, N = 16 centers, K = 4 x 32
//      dims, u8 x u8 -> s32, exact) into this CTA's TMEM columns;
//   3. warp w reads the dot products of rows 32w..32w+31 (its TMEM lane quarter) and takes the
//      argmin of |c_b|^2 - 2 x.c_b, lowest index on ties (kmeans.cu:131-135), updating the
//      assignment, the per-center counts and the changed count;
//   4. the same warp adds its rows into the node's per-CTA center sums: lane l owns dims
//      4l..4l+3 and adds each row's four bytes with shared atomics, the sums stored
//      dim-interleaved so that the 32 lanes hit 32 banks.
// Counts and sums go to global memory when the CTA moves to another node.  Several CTAs per SM
// overlap one another's gathers, MMAs and sums.
constexpr uint32_t kAssignThreads = 128;
constexpr uint32_t kAssignRows = 128;
constexpr uint32_t kAssignTmemCols = 32; // the smallest allocation; the MMA writes 16 columns
constexpr uint32_t kAssignCtasPerSm = 8; // by registers (<= 64) and shared memory; 256 TMEM columns

struct AssignSmem {
    uint8_t tile[kAssignRows * kDims];   // member rows, 128-byte swizzle (1024-byte aligned)
    uint8_t cen[kMaxBranch * kDims];     // node centers, same layout
    uint32_t acc[kMaxBranch * kDims];    // center sums of the current node, see accIndex
    int32_t cn[kMaxBranch];
    uint32_t cnt[kMaxBranch];
    uint8_t bsel[kAssignRows];
    uint64_t mmaBar;
    uint32_t tmemBase;
    uint32_t chg;
    uint32_t abortFlag;
};
constexpr size_t kAssignSmemBytes = sizeof(AssignSmem) + 1024;

// Position of (center b, dim d = 4 l + k) in AssignSmem::acc: b * 128 + 32 k + l.
__device__ __forceinline__ uint32_t accIndex(uint32_t b, uint32_t d)
{
    return b * kDims + (d & 3u) * 32u + (d >> 2);
}

__global__ void __launch_bounds__(kAssignThreads, kAssignCtasPerSm) assignKernel(KMeansLevel lv, const NodeTile* tiles,
                                                                  const uint32_t* nTilesDev)
{
    extern __shared__ uint8_t smemRaw[];
    AssignSmem& S = *reinterpret_cast<AssignSmem*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    const uint32_t tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
    const uint32_t T = *nTilesDev;
    const uint32_t t0 = static_cast<uint32_t>(uint64_t(T) * blockIdx.x / gridDim.x);
    const uint32_t t1 = static_cast<uint32_t>(uint64_t(T) * (blockIdx.x + 1) / gridDim.x);
    volatile uint32_t* abortFlag = &S.abortFlag;
    if (tid == 0) {
        mbarInit(&S.mmaBar, 1);
        S.abortFlag = 0;
        fenceMbarInit();
    }
    if (warp == 0) {
        tmemAlloc(&S.tmemBase, kAssignTmemCols);
        tmemRelinquish();
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = S.tmemBase;
    uint32_t curNode = 0xFFFFFFFFu, phase = 0;
    bool curExclusive = false; // every tile of the current node is in this CTA's range
    auto flush = [&]() {
        __syncthreads();
        if (curNode != 0xFFFFFFFFu) {
            // A node no other CTA touches in this launch is written with plain stores (its
            // global accumulators are zero on entry); a shared node is added atomically.
            for (uint32_t i = tid; i < kMaxBranch * kDims; i += kAssignThreads) {
                const uint32_t b = i / kDims, d = i % kDims;
                const uint32_t v = S.acc[accIndex(b, d)];
                unsigned long long* dst = lv.sums + (uint64_t(curNode) * kMaxBranch + b) * kDims + d;
                if (v) {
                    if (curExclusive) *dst = v;
                    else atomicAdd(dst, (unsigned long long)v);
                }
            }
            if (tid < kMaxBranch && S.cnt[tid]) {
                uint32_t* dst = lv.counts + uint64_t(curNode) * kMaxBranch + tid;
                if (curExclusive) *dst = S.cnt[tid];
                else atomicAdd(dst, S.cnt[tid]);
            }
            if (tid == 0 && S.chg) {
                if (curExclusive) lv.changed[curNode] = S.chg;
                else atomicAdd(lv.changed + curNode, S.chg);
            }
        }
        __syncthreads();
    };
    for (uint32_t t = t0; t < t1; t++) {
        const NodeTile ti = tiles[t];
        if (lv.lastChanged[ti.node] == 0) continue; // frozen node (kmeans.cu:238-240)
        if (ti.node != curNode) {
            flush();
            curNode = ti.node;
            curExclusive = ti.first >= t0 && uint64_t(ti.first) + (lv.nodeCnt[curNode] + kAssignRows - 1) / kAssignRows <= t1;
            {
                // thread i copies chunk i % 8 of center i / 8 (16 centers x 8 chunks)
                const uint32_t b = tid / 8, c = tid % 8;
                const uint4 v = reinterpret_cast<const uint4*>(lv.centers + (uint64_t(curNode) * kMaxBranch + b) * kDims)[c];
                *reinterpret_cast<uint4*>(S.cen + b * kDims + ((c ^ (b & 7u)) << 4)) = v;
            }
            if (tid < kMaxBranch) {
                S.cn[tid] = lv.cnorm[uint64_t(curNode) * kMaxBranch + tid];
                S.cnt[tid] = 0;
            }
            for (uint32_t i = tid; i < kMaxBranch * kDims; i += kAssignThreads) S.acc[i] = 0;
            if (tid == 0) S.chg = 0;
        }
        {
            // eight threads per row, 16 rows per round; rows past the tile's count repeat its
            // first member (their results are not used)
            const uint32_t c = tid % 8;
            uint32_t m[kAssignRows / 16];
#pragma unroll
            for (uint32_t k = 0; k < kAssignRows / 16; k++) {
                const uint32_t row = 16u * k + tid / 8;
                m[k] = lv.members[uint64_t(ti.start) + (row < ti.count ? row : 0u)];
            }
#pragma unroll
            for (uint32_t k = 0; k < kAssignRows / 16; k++) {
                const uint32_t row = 16u * k + tid / 8;
                cpAsync16(S.tile + row * kDims + ((c ^ (row & 7u)) << 4), lv.desc + uint64_t(m[k]) * kDims + (c << 4));
            }
            cpAsyncCommit();
            cpAsyncWait<0>();
        }
        // the copies and the center stores are generic-proxy writes read by the tensor core
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tcFenceAfter();
            const uint32_t aBase = smemAddr(S.tile), bBase = smemAddr(S.cen);
#pragma unroll
            for (uint32_t q4 = 0; q4 < 4; q4++)
                mmaU8(tmem, smemDescSw128(aBase + 32u * q4), smemDescSw128(bBase + 32u * q4), idescU8(16),
                      q4 > 0 ? 1u : 0u);
            mmaCommit(&S.mmaBar);
        }
        if (!mbarWait(&S.mmaBar, phase, abortFlag, lv.err, 40)) break;
        phase ^= 1u;
        tcFenceAfter();
        const uint32_t row = tid; // warp w reads TMEM lanes 32w .. 32w + 31
        uint32_t r[16];
        tmemLoad16(tmem + ((warp * 32u) << 16), r);
        tmemWaitTie(r);
        tcFenceBefore(); // the next step's MMA overwrites these columns after the barriers below
        int32_t best = S.cn[0] - 2 * static_cast<int32_t>(r[0]);
        uint32_t bi = 0;
#pragma unroll
        for (uint32_t b = 1; b < kMaxBranch; b++) {
            const int32_t sc = S.cn[b] - 2 * static_cast<int32_t>(r[b]);
            if (sc < best) {
                best = sc;
                bi = b;
            }
        }
        if (row < ti.count) {
            const uint64_t at = uint64_t(ti.start) + row;
            if (lv.assign[at] != bi) atomicAdd(&S.chg, 1u);
            lv.assign[at] = static_cast<uint8_t>(bi);
            atomicAdd(&S.cnt[bi], 1u);
        }
        S.bsel[row] = static_cast<uint8_t>(bi);
        __syncwarp();
        const uint32_t rEnd = ti.count < 32u * warp + 32u ? ti.count : 32u * warp + 32u;
        for (uint32_t rr = 32u * warp; rr < rEnd; rr++) {
            const uint32_t b = S.bsel[rr];
            const uint32_t x = *reinterpret_cast<const uint32_t*>(S.tile + rr * kDims + (((lane >> 2) ^ (rr & 7u)) << 4) +
                                                                  ((lane & 3u) << 2));
            uint32_t* a = S.acc + b * kDims + lane;
            atomicAdd(a, x & 0xFFu);
            atomicAdd(a + 32, (x >> 8) & 0xFFu);
            atomicAdd(a + 64, (x >> 16) & 0xFFu);
            atomicAdd(a + 96, x >> 24);
        }
        __syncthreads(); // the tile and bsel are rewritten by the next step
    }
    flush();
    if (warp == 0) {
        tcFenceAfter();
        tmemDealloc(tmem, kAssignTmemCols);
    }
}

// ------------------------------------------------------------------ assign, sums on the tensor core
// The same assignment as assignKernel; the center sums come from a second MMA per tile instead of
// 128 shared atomics per member: D[dim][center] += XT[dim][member] * OH[center][member], with XT
// the tile transposed in shared memory (4 x 4 byte blocks through byte permutes) and OH the
// one-hot of the members' centers built from ballots.  Both operands are K-major with K =
// members, u8 x u8 -> s32 (exact); D lives in TMEM columns [16, 32) and accumulates over the
// node's tiles in this CTA, read and written out when the CTA moves to another node (or every
// kTsFlushTiles tiles, which keeps each s32 below 2^31: 65,536 x 128 x 255 < 2^31).
constexpr uint32_t kAssignTsCtasPerSm = 4;     // by shared memory (~54 KB each)
constexpr uint32_t kTsFlushTiles = 65536;
constexpr uint32_t kTsTileWindow = kAssignThreads; // one tile entry per thread per refill
constexpr uint32_t kTsFrozen = 0x80000000u;

struct AssignTsSmem {
    uint8_t tile[2][kAssignRows * kDims]; // member rows, K-major (dims), 128-byte swizzle; the
                                          // next tile's rows are gathered while this one is scored
    uint8_t xt[kDims * kAssignRows];     // the rows transposed: [dim][member], same layout
    uint8_t oh[kMaxBranch * kAssignRows]; // [center][member]: 1 where the member chose the center
    uint8_t cen[kMaxBranch * kDims];     // node centers
    NodeTile win[kTsTileWindow];         // tiles [winBase, winBase + kTsTileWindow) of the CTA's
                                         // range, count | kTsFrozen for a frozen node
    int32_t cn[kMaxBranch];
    uint32_t cnt[kMaxBranch];
    uint64_t mmaBar, sumBar;
    uint32_t tmemBase;
    uint32_t chg;
    uint32_t abortFlag;
};
constexpr size_t kAssignTsSmemBytes = sizeof(AssignTsSmem) + 1024;

// Byte (row, col) of a 128-column, 128-byte-swizzled K-major operand.
__device__ __forceinline__ uint32_t sw128(uint32_t row, uint32_t col)
{
    return row * 128u + ((((col >> 4) ^ row) & 7u) << 4) + (col & 15u);
}

__global__ void __launch_bounds__(kAssignThreads, kAssignTsCtasPerSm)
    assignKernelTs(KMeansLevel lv, const NodeTile* tiles, const uint32_t* nTilesDev)
{
    extern __shared__ uint8_t smemRaw[];
    AssignTsSmem& S =
        *reinterpret_cast<AssignTsSmem*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    const uint32_t tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
    const uint32_t T = *nTilesDev;
    const uint32_t t0 = static_cast<uint32_t>(uint64_t(T) * blockIdx.x / gridDim.x);
    const uint32_t t1 = static_cast<uint32_t>(uint64_t(T) * (blockIdx.x + 1) / gridDim.x);
    volatile uint32_t* abortFlag = &S.abortFlag;
    if (tid == 0) {
        mbarInit(&S.mmaBar, 1);
        mbarInit(&S.sumBar, 1);
        S.abortFlag = 0;
        fenceMbarInit();
    }
    if (warp == 0) {
        tmemAlloc(&S.tmemBase, kAssignTmemCols);
        tmemRelinquish();
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = S.tmemBase;
    uint32_t curNode = 0xFFFFFFFFu, phase = 0, sumPhase = 0, accTiles = 0, buf = 0;
    bool curExclusive = false, sumInFlight = false, ok = true;
    // The tile list and the frozen flags are read a window of kTsTileWindow tiles at a time (one
    // load per thread, all in flight together), so that finding the next live tile costs no
    // global round trip; the member indices of the next tile are loaded into registers one
    // tile ahead of its row copies.  Every thread runs the same window refills (uniform).
    uint32_t winBase = t0;
    auto refill = [&](uint32_t base) {
        __syncthreads(); // nobody reads the old window any more
        if (base + tid < t1) {
            NodeTile x = tiles[base + tid];
            if (lv.lastChanged[x.node] == 0) x.count |= kTsFrozen; // frozen node (kmeans.cu:238-240)
            S.win[tid] = x;
        }
        winBase = base;
        __syncthreads();
    };
    auto entry = [&](uint32_t t) -> NodeTile {
        if (t - winBase >= kTsTileWindow) refill(t);
        return S.win[t - winBase];
    };
    // the first live tile at or after t, or t1
    auto nextLive = [&](uint32_t t) -> uint32_t {
        for (; t < t1; t++)
            if (!(entry(t).count & kTsFrozen)) return t;
        return t1;
    };
    auto loadIndices = [&](const NodeTile& tn, uint32_t (&m)[kAssignRows / 16]) {
#pragma unroll
        for (uint32_t k = 0; k < kAssignRows / 16; k++) {
            const uint32_t row = 16u * k + tid / 8;
            m[k] = lv.members[uint64_t(tn.start) + (row < tn.count ? row : 0u)];
        }
    };
    // eight threads per row, 16 rows per round; rows past the tile's count repeat its first
    // member (their results are not used); one copy group per tile
    auto gatherRows = [&](const uint32_t (&m)[kAssignRows / 16], uint32_t b) {
        const uint32_t c = tid % 8;
#pragma unroll
        for (uint32_t k = 0; k < kAssignRows / 16; k++) {
            const uint32_t row = 16u * k + tid / 8;
            cpAsync16(S.tile[b] + row * kDims + ((c ^ (row & 7u)) << 4), lv.desc + uint64_t(m[k]) * kDims + (c << 4));
        }
        cpAsyncCommit();
    };
    auto waitSums = [&]() {
        if (!sumInFlight) return;
        ok = ok && mbarWait(&S.sumBar, sumPhase, abortFlag, lv.err, 42);
        sumPhase ^= 1u;
        sumInFlight = false;
        tcFenceAfter();
    };
    // writes the node's partial sums (TMEM), counts and change count
    auto flush = [&]() {
        __syncthreads();
        if (curNode != 0xFFFFFFFFu) {
            if (accTiles > 0) {
                waitSums();
                uint32_t r[16];
                tmemLoad16(tmem + 16u + ((warp * 32u) << 16), r); // lane = dimension tid
                tmemWaitTie(r);
                tcFenceBefore();
#pragma unroll
                for (uint32_t b = 0; b < kMaxBranch; b++) {
                    if (r[b] == 0) continue;
                    unsigned long long* dst = lv.sums + (uint64_t(curNode) * kMaxBranch + b) * kDims + tid;
                    if (curExclusive) *dst = r[b];
                    else atomicAdd(dst, (unsigned long long)r[b]);
                }
            }
            if (tid < kMaxBranch && S.cnt[tid]) {
                uint32_t* dst = lv.counts + uint64_t(curNode) * kMaxBranch + tid;
                if (curExclusive) *dst = S.cnt[tid];
                else atomicAdd(dst, S.cnt[tid]);
            }
            if (tid == 0 && S.chg) {
                if (curExclusive) lv.changed[curNode] = S.chg;
                else atomicAdd(lv.changed + curNode, S.chg);
            }
        }
        accTiles = 0;
        __syncthreads();
    };
    if (t0 < t1) refill(t0);
    uint32_t t = nextLive(t0);
    NodeTile ti{}, tn1{};
    uint32_t mNext[kAssignRows / 16];
    if (t < t1) {
        ti = entry(t);
        loadIndices(ti, mNext);
        gatherRows(mNext, buf);
    }
    uint32_t n1 = t < t1 ? nextLive(t + 1) : t1;
    if (n1 < t1) {
        tn1 = entry(n1);
        loadIndices(tn1, mNext);
    }
    while (ok && t < t1) {
        if (ti.node != curNode) {
            flush();
            curNode = ti.node;
            curExclusive = ti.first >= t0 && uint64_t(ti.first) + (lv.nodeCnt[curNode] + kAssignRows - 1) / kAssignRows <= t1;
            {
                const uint32_t b = tid / 8, c = tid % 8;
                const uint4 v = reinterpret_cast<const uint4*>(lv.centers + (uint64_t(curNode) * kMaxBranch + b) * kDims)[c];
                *reinterpret_cast<uint4*>(S.cen + b * kDims + ((c ^ (b & 7u)) << 4)) = v;
            }
            if (tid < kMaxBranch) {
                S.cn[tid] = lv.cnorm[uint64_t(curNode) * kMaxBranch + tid];
                S.cnt[tid] = 0;
            }
            if (tid == 0) S.chg = 0;
        } else if (accTiles == kTsFlushTiles) {
            // keep each s32 sum below 2^31: add this node's partial results to global memory and
            // go on from zero (its later flushes add too)
            curExclusive = false;
            flush();
            if (tid < kMaxBranch) S.cnt[tid] = 0;
            if (tid == 0) S.chg = 0;
            __syncthreads();
        }
        // the next live tile's rows go into the other buffer (its indices were loaded one tile
        // ago), the indices of the one after it into registers; then this tile's rows must be in
        uint32_t n2 = t1;
        NodeTile tn2{};
        if (n1 < t1) {
            gatherRows(mNext, buf ^ 1u);
            n2 = nextLive(n1 + 1);
            if (n2 < t1) {
                tn2 = entry(n2);
                loadIndices(tn2, mNext);
            }
            cpAsyncWait<1>();
        } else {
            cpAsyncWait<0>();
        }
        const uint32_t row = tid;
        const bool valid = row < ti.count;
        const uint64_t at = uint64_t(ti.start) + row;
        const uint32_t prevAssign = valid ? lv.assign[at] : 0u;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        const uint8_t* tileBuf = S.tile[buf];
        if (tid == 0) {
            tcFenceAfter();
            const uint32_t aBase = smemAddr(tileBuf), bBase = smemAddr(S.cen);
#pragma unroll
            for (uint32_t q4 = 0; q4 < 4; q4++)
                mmaU8(tmem, smemDescSw128(aBase + 32u * q4), smemDescSw128(bBase + 32u * q4), idescU8(16),
                      q4 > 0 ? 1u : 0u);
            mmaCommit(&S.mmaBar);
        }
        if (!mbarWait(&S.mmaBar, phase, abortFlag, lv.err, 41)) {
            ok = false;
            break;
        }
        phase ^= 1u;
        tcFenceAfter();
        uint32_t r[16];
        tmemLoad16(tmem + ((warp * 32u) << 16), r);
        tmemWaitTie(r);
        tcFenceBefore();
        int32_t best = S.cn[0] - 2 * static_cast<int32_t>(r[0]);
        uint32_t bi = 0;
#pragma unroll
        for (uint32_t b = 1; b < kMaxBranch; b++) {
            const int32_t sc = S.cn[b] - 2 * static_cast<int32_t>(r[b]);
            if (sc < best) {
                best = sc;
                bi = b;
            }
        }
        if (valid) {
            if (prevAssign != bi) atomicAdd(&S.chg, 1u);
            lv.assign[at] = static_cast<uint8_t>(bi);
            atomicAdd(&S.cnt[bi], 1u);
        }
        // the previous tile's sums MMA must be done reading xt and oh before they are rewritten
        waitSums();
        if (!ok) break;
        // one-hot: lane c writes row c's 32 bytes of this warp's members (bit i = member 32 w + i)
        uint32_t mine = 0;
#pragma unroll
        for (uint32_t c = 0; c < kMaxBranch; c++) {
            const uint32_t bits = __ballot_sync(0xFFFFFFFFu, valid && bi == c);
            if (lane == c) mine = bits;
        }
        if (lane < kMaxBranch) {
#pragma unroll
            for (uint32_t half = 0; half < 2; half++) {
                uint32_t w4[4];
#pragma unroll
                for (uint32_t q = 0; q < 4; q++) {
                    const uint32_t nib = (mine >> (16u * half + 4u * q)) & 0xFu;
                    w4[q] = (nib & 1u) | ((nib & 2u) << 7) | ((nib & 4u) << 14) | ((nib & 8u) << 21);
                }
                const uint32_t col = 32u * warp + 16u * half;
                *reinterpret_cast<uint4*>(S.oh + sw128(lane, col)) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
            }
        }
        // transpose this warp's 32 rows into xt columns 32 w .. 32 w + 31, 4 x 4 byte blocks:
        // lane = (dimension quad dq0 = lane / 8, member quad mq = lane % 8), eight dimension quads
        {
            const uint32_t m0 = 32u * warp + 4u * (lane & 7u);
#pragma unroll
            for (uint32_t k = 0; k < 8; k++) {
                const uint32_t d0 = 4u * ((lane >> 3) + 4u * k);
                const uint32_t w0 = *reinterpret_cast<const uint32_t*>(tileBuf + sw128(m0, d0));
                const uint32_t w1 = *reinterpret_cast<const uint32_t*>(tileBuf + sw128(m0 + 1, d0));
                const uint32_t w2 = *reinterpret_cast<const uint32_t*>(tileBuf + sw128(m0 + 2, d0));
                const uint32_t w3 = *reinterpret_cast<const uint32_t*>(tileBuf + sw128(m0 + 3, d0));
                const uint32_t a = __byte_perm(w0, w1, 0x5140), b = __byte_perm(w2, w3, 0x5140);
                const uint32_t c = __byte_perm(w0, w1, 0x7362), d = __byte_perm(w2, w3, 0x7362);
                *reinterpret_cast<uint32_t*>(S.xt + sw128(d0, m0)) = __byte_perm(a, b, 0x5410);
                *reinterpret_cast<uint32_t*>(S.xt + sw128(d0 + 1, m0)) = __byte_perm(a, b, 0x7632);
                *reinterpret_cast<uint32_t*>(S.xt + sw128(d0 + 2, m0)) = __byte_perm(c, d, 0x5410);
                *reinterpret_cast<uint32_t*>(S.xt + sw128(d0 + 3, m0)) = __byte_perm(c, d, 0x7632);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads(); // xt, oh complete; the tile is rewritten by the next gather
        if (tid == 0) {
            tcFenceAfter();
            const uint32_t aBase = smemAddr(S.xt), bBase = smemAddr(S.oh);
#pragma unroll
            for (uint32_t q4 = 0; q4 < 4; q4++)
                mmaU8(tmem + 16u, smemDescSw128(aBase + 32u * q4), smemDescSw128(bBase + 32u * q4), idescU8(16),
                      (accTiles > 0 || q4 > 0) ? 1u : 0u);
            mmaCommit(&S.sumBar);
        }
        sumInFlight = true;
        accTiles++;
        buf ^= 1u;
        t = n1;
        ti = tn1;
        n1 = n2;
        tn1 = tn2;
    }
    cpAsyncWait<0>(); // a prefetch of a tile that was not scored (abort) must land before exit
    if (ok) flush();
    else waitSums();
    if (warp == 0) {
        tcFenceAfter();
        tmemDealloc(tmem, kAssignTmemCols);
    }
}

// ------------------------------------------------------------------ regroup
constexpr uint32_t kRegroupRows = 32;

__global__ void regroupHistKernel(KMeansLevel lv, const NodeTile* tiles, const uint32_t* nTilesDev, uint32_t maxTiles,
                                  uint32_t* tileHist)
{
    // warp per 32-member tile: lane q < B writes how many members chose center q
    const uint32_t T = *nTilesDev;
    const uint32_t warpsTotal = gridDim.x * (blockDim.x / 32);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t t = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; t < T; t += warpsTotal) {
        const NodeTile ti = tiles[t];
        const uint32_t b = lane < ti.count ? lv.assign[ti.start + lane] : 0xFFu;
        uint32_t c = 0;
        for (uint32_t q = 0; q < lv.B; q++) {
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, b == q);
            if (lane == q) c = __popc(m);
        }
        if (lane < lv.B) tileHist[uint64_t(lane) * maxTiles + t] = c;
    }
}

__global__ void regroupChildKernel(KMeansLevel lv, const uint32_t* tileOffNode, uint32_t maxTiles,
                                   const uint32_t* tileHist, const uint32_t* tileScan, uint32_t* childCnt,
                                   uint32_t* childOff)
{
    // thread per node: child sizes from the per-center scans over the node's tiles, children
    // laid out in center order (Vocabulary.cpp:83-98)
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= lv.nbNodes) return;
    const uint32_t first = tileOffNode[g];
    const uint32_t nt = (lv.nodeCnt[g] + kRegroupRows - 1) / kRegroupRows;
    uint32_t off = lv.nodeOff[g];
    for (uint32_t b = 0; b < lv.B; b++) {
        uint32_t c = 0;
        if (nt) {
            const uint64_t row = uint64_t(b) * maxTiles;
            const uint32_t lastT = first + nt - 1;
            c = tileScan[row + lastT] - tileScan[row + first] + tileHist[row + lastT];
        }
        childCnt[uint64_t(g) * lv.B + b] = c;
        childOff[uint64_t(g) * lv.B + b] = off;
        off += c;
    }
}

__global__ void regroupScatterKernel(KMeansLevel lv, const NodeTile* tiles, const uint32_t* nTilesDev,
                                     uint32_t maxTiles, const uint32_t* tileScan, const uint32_t* childOff,
                                     uint32_t* childMembers)
{
    const uint32_t T = *nTilesDev;
    const uint32_t warpsTotal = gridDim.x * (blockDim.x / 32);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t t = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; t < T; t += warpsTotal) {
        const NodeTile ti = tiles[t];
        const bool valid = lane < ti.count;
        const uint32_t b = valid ? lv.assign[ti.start + lane] : 0xFFu;
        const uint32_t same = __match_any_sync(0xFFFFFFFFu, b);
        const uint32_t rank = __popc(same & ((1u << lane) - 1u));
        if (valid) {
            const uint64_t row = uint64_t(b) * maxTiles;
            const uint32_t within = tileScan[row + t] - tileScan[row + ti.first];
            const uint32_t dst = childOff[uint64_t(ti.node) * lv.B + b] + within + rank;
            childMembers[dst] = lv.members[ti.start + lane];
        }
    }
}

} // namespace

size_t scanTempWords(uint64_t n)
{
    const uint64_t blocks = (n + kScanTile - 1) / kScanTile;
    return blocks + 32;
}

void exclusiveScanU32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* tmp, cudaStream_t s)
{
    if (n == 0) return;
    const uint32_t blocks = static_cast<uint32_t>((n + kScanTile - 1) / kScanTile);
    scanBlockSums<<<blocks, kScanBlock, 0, s>>>(in, n, tmp);
    scanSingle<<<1, kScanBlock, 0, s>>>(tmp, blocks);
    scanApply<<<blocks, kScanBlock, 0, s>>>(in, n, tmp, out);
    RBW_CUDA(cudaGetLastError());
}

void buildNodeTiles(const uint32_t* nodeCnt, const uint32_t* nodeOff, uint32_t nbNodes, uint32_t tileRows,
                    uint32_t* tileOff, uint32_t* tmp, NodeTile* tiles, uint32_t maxTiles, uint32_t* totals,
                    cudaStream_t s)
{
    ceilDivKernel<<<(nbNodes + 255) / 256, 256, 0, s>>>(nodeCnt, nbNodes, tileRows, tileOff);
    exclusiveScanU32(tileOff, tileOff, nbNodes, tmp, s);
    tilesTotal<<<1, 1, 0, s>>>(nodeCnt, tileOff, nbNodes, tileRows, totals);
    const uint32_t blocks = std::min<uint32_t>((maxTiles + 255) / 256, 8192);
    fillNodeTiles<<<std::max(blocks, 1u), 256, 0, s>>>(nodeCnt, nodeOff, tileOff, nbNodes, tileRows, totals, maxTiles,
                                                      tiles);
    RBW_CUDA(cudaGetLastError());
}

void launchInitCenters(const KMeansLevel& lv, const uint32_t* pos, uint64_t nbDescTotal, cudaStream_t s)
{
    const uint64_t total = uint64_t(lv.nbNodes) * kMaxBranch * 8;
    initCentersKernel<<<static_cast<uint32_t>((total + 255) / 256), 256, 0, s>>>(lv, pos, nbDescTotal, 0);
    RBW_CUDA(cudaGetLastError());
}

void launchInitCentersFromDesc(const KMeansLevel& lv, const uint32_t* descIdx, uint64_t nbDescTotal, cudaStream_t s)
{
    const uint64_t total = uint64_t(lv.nbNodes) * kMaxBranch * 8;
    initCentersKernel<<<static_cast<uint32_t>((total + 255) / 256), 256, 0, s>>>(lv, descIdx, nbDescTotal, 1);
    RBW_CUDA(cudaGetLastError());
}

void launchCenterNorms(const KMeansLevel& lv, cudaStream_t s)
{
    const uint64_t total = uint64_t(lv.nbNodes) * kMaxBranch;
    centerNormsKernel<<<static_cast<uint32_t>((total + 255) / 256), 256, 0, s>>>(lv);
    RBW_CUDA(cudaGetLastError());
}

void launchKMeansPPInit(const KMeansLevel& lv, uint64_t seed, uint32_t level, uint32_t* nValid, cudaStream_t s)
{
    kmeansPPKernel<<<lv.nbNodes, kPPSample, 0, s>>>(lv, seed, level, nValid);
    RBW_CUDA(cudaGetLastError());
}

void launchAssign(const KMeansLevel& lv, const NodeTile* tiles, const uint32_t* nTilesDev, uint32_t maxTiles,
                  cudaStream_t s)
{
    int dev = 0, sms = 0;
    RBW_CUDA(cudaGetDevice(&dev));
    RBW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // A fixed grid (the occupancy query gave one CTA per SM on some launches, 3-4x slower) of
    // up to kAssignCtasPerSm CTAs per SM, the count the autotuner chose for this workload.
    static_assert(kAssignCtasPerSm * kAssignTmemCols <= 512, "TMEM columns of the resident CTAs");
    static_assert(kAssignCtasPerSm * kAssignSmemBytes <= 227 * 1024, "shared memory of the resident CTAs");
    static_assert(kAssignTsCtasPerSm * kAssignTsSmemBytes <= 227 * 1024, "shared memory of the resident CTAs");
    const bool tensorSums = tunedValue(kTuneAssignSums, lv.B, 0, lv.nbMembers) == 2;
    const uint32_t cap = tensorSums ? kAssignTsCtasPerSm : kAssignCtasPerSm;
    const uint32_t perSm = std::min(cap, tunedValue(kTuneAssignCtasPerSm, lv.B, 0, lv.nbMembers));
    const uint32_t grid = std::max(1u, std::min<uint32_t>(maxTiles, static_cast<uint32_t>(sms) * perSm));
    ScopedKernelTimer timer(kTimedAssign, s);
    if (tensorSums) {
        static std::atomic<uint64_t> attr{0};
        setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(assignKernelTs), int(kAssignTsSmemBytes), attr);
        assignKernelTs<<<grid, kAssignThreads, kAssignTsSmemBytes, s>>>(lv, tiles, nTilesDev);
    } else {
        assignKernel<<<grid, kAssignThreads, kAssignSmemBytes, s>>>(lv, tiles, nTilesDev);
    }
    RBW_CUDA(cudaGetLastError());
}

void launchRegroup(const KMeansLevel& lv, const RegroupScratch& rs, uint32_t* childMembers, uint32_t* childCnt,
                   uint32_t* childOff, cudaStream_t s)
{
    buildNodeTiles(lv.nodeCnt, lv.nodeOff, lv.nbNodes, kRegroupRows, rs.tileOff, rs.scanTmp, rs.tiles, rs.maxTiles,
                   rs.totals, s);
    RBW_CUDA(cudaMemsetAsync(rs.tileHist, 0, sizeof(uint32_t) * uint64_t(lv.B) * rs.maxTiles, s));
    const uint32_t warpsPerBlock = 8;
    const uint32_t blocks = std::max(1u, std::min<uint32_t>((rs.maxTiles + warpsPerBlock - 1) / warpsPerBlock, 16384));
    regroupHistKernel<<<blocks, 32 * warpsPerBlock, 0, s>>>(lv, rs.tiles, rs.totals, rs.maxTiles, rs.tileHist);
    exclusiveScanU32(rs.tileHist, rs.tileScan, uint64_t(lv.B) * rs.maxTiles, rs.scanTmp, s);
    regroupChildKernel<<<(lv.nbNodes + 255) / 256, 256, 0, s>>>(lv, rs.tileOff, rs.maxTiles, rs.tileHist,
                                                                rs.tileScan, childCnt, childOff);
    regroupScatterKernel<<<blocks, 32 * warpsPerBlock, 0, s>>>(lv, rs.tiles, rs.totals, rs.maxTiles, rs.tileScan,
                                                                childOff, childMembers);
    RBW_CUDA(cudaGetLastError());
}

} // namespace rbw
