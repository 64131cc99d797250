// Hierarchical k-means kernels.  Distances are exact integers: score_b = |c_b|^2 - 2 x.c_b with
// x.c_b from dp4a (u8 x u8 -> u32), argmin with the lowest index on ties (kmeans.cu:131-135).
// Center sums are exact (u32 in shared memory, u64 in global memory).
#include "kmeans.cuh"
#include "timing.h"

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
__device__ __forceinline__ uint64_t splitmix64(uint64_t& s)
{
    // SplitMix64 (Steele, Lea, Flood 2014).
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint32_t dist128Dev(const uint8_t* a, const uint8_t* b)
{
    const uint4* a4 = reinterpret_cast<const uint4*>(a);
    const uint4* b4 = reinterpret_cast<const uint4*>(b);
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint4 x = a4[k], y = b4[k];
        const uint32_t d0 = __vabsdiffu4(x.x, y.x), d1 = __vabsdiffu4(x.y, y.y);
        const uint32_t d2 = __vabsdiffu4(x.z, y.z), d3 = __vabsdiffu4(x.w, y.w);
        acc = __dp4a(d0, d0, acc);
        acc = __dp4a(d1, d1, acc);
        acc = __dp4a(d2, d2, acc);
        acc = __dp4a(d3, d3, acc);
    }
    return acc;
}

constexpr uint32_t kPPSample = 256;

// One CTA (256 threads) per node.  Same specification as the oracle's orc_kmeanspp_init:
// SplitMix64 stream seeded by (seed, level, node); Floyd sampling of min(n, 256) member
// positions (sorted); first center uniform; then D^2 sampling with exact integer weights.
__global__ void __launch_bounds__(kPPSample) kmeansPPKernel(KMeansLevel lv, uint64_t seed, uint32_t level,
                                                            uint32_t* nValidOut)
{
    __shared__ uint32_t pos[kPPSample];
    __shared__ uint32_t cand[kPPSample];
    __shared__ unsigned long long d2[kPPSample];
    __shared__ unsigned long long pre[kPPSample];
    __shared__ uint32_t chosen[kMaxBranch];
    __shared__ uint32_t nChosen;
    __shared__ unsigned long long tPick;
    __shared__ uint64_t rngState;
    const uint32_t g = blockIdx.x;
    const uint32_t n = lv.nodeCnt[g];
    const uint32_t tid = threadIdx.x;
    const uint32_t S = n < kPPSample ? n : kPPSample;
    if (tid == 0) {
        uint64_t s = seed ^ (uint64_t(level) * 0x9E3779B97F4A7C15ull) ^ (uint64_t(g) * 0xD1B54A32D192ED03ull);
        if (n > kPPSample) {
            uint32_t m = 0;
            for (uint32_t j = n - S; j < n; j++) {
                const uint32_t t = static_cast<uint32_t>(splitmix64(s) % (uint64_t(j) + 1));
                bool found = false;
                for (uint32_t q = 0; q < m; q++) found |= (pos[q] == t);
                pos[m++] = found ? j : t;
            }
            // insertion sort (<= 256 entries)
            for (uint32_t a = 1; a < m; a++) {
                const uint32_t v = pos[a];
                int32_t q = int32_t(a) - 1;
                while (q >= 0 && pos[q] > v) {
                    pos[q + 1] = pos[q];
                    q--;
                }
                pos[q + 1] = v;
            }
        }
        rngState = s;
        nChosen = 0;
    }
    __syncthreads();
    if (n == 0) {
        if (tid == 0) nValidOut[g] = 0;
        for (uint32_t i = tid; i < kMaxBranch * 8; i += blockDim.x) {
            reinterpret_cast<uint4*>(lv.centers + uint64_t(g) * kMaxBranch * kDims)[i] =
                make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        }
        return;
    }
    if (tid < S) cand[tid] = lv.members[lv.nodeOff[g] + (n > kPPSample ? pos[tid] : tid)];
    __syncthreads();
    if (tid == 0) {
        uint64_t s = rngState;
        chosen[0] = static_cast<uint32_t>(splitmix64(s) % S);
        rngState = s;
        nChosen = 1;
    }
    __syncthreads();
    if (tid < S) d2[tid] = dist128Dev(lv.desc + uint64_t(cand[tid]) * kDims, lv.desc + uint64_t(cand[chosen[0]]) * kDims);
    __syncthreads();
    for (uint32_t k = 1; k < lv.B; k++) {
        // inclusive prefix of d2 (Hillis-Steele in shared memory)
        if (tid < kPPSample) pre[tid] = tid < S ? d2[tid] : 0ull;
        __syncthreads();
        for (uint32_t off = 1; off < kPPSample; off <<= 1) {
            unsigned long long v = 0;
            if (tid >= off) v = pre[tid - off];
            __syncthreads();
            pre[tid] += v;
            __syncthreads();
        }
        const unsigned long long total = pre[S - 1];
        if (total == 0) break; // uniform across the CTA
        if (tid == 0) {
            uint64_t s = rngState;
            tPick = splitmix64(s) % total;
            rngState = s;
        }
        __syncthreads();
        // smallest i with pre[i] > t
        if (tid < S) {
            const bool hit = pre[tid] > tPick && (tid == 0 || pre[tid - 1] <= tPick);
            if (hit) {
                chosen[k] = tid;
                nChosen = k + 1;
            }
        }
        __syncthreads();
        if (tid < S) {
            const uint32_t d = dist128Dev(lv.desc + uint64_t(cand[tid]) * kDims, lv.desc + uint64_t(cand[chosen[k]]) * kDims);
            if (d < d2[tid]) d2[tid] = d;
        }
        __syncthreads();
    }
    const uint32_t nv = nChosen;
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
constexpr uint32_t kAssignThreads = 128;

__global__ void __launch_bounds__(kAssignThreads) assignKernel(KMeansLevel lv, const NodeTile* tiles,
                                                               const uint32_t* nTilesDev)
{
    __shared__ uint4 cs[kMaxBranch][8];       // node centers
    __shared__ int32_t cn[kMaxBranch];
    __shared__ uint32_t acc[kMaxBranch][kDims + 4]; // per-CTA center sums (padded rows)
    __shared__ uint32_t cnt[kMaxBranch];
    __shared__ uint32_t chg;
    const uint32_t T = *nTilesDev;
    const uint32_t t0 = static_cast<uint32_t>(uint64_t(T) * blockIdx.x / gridDim.x);
    const uint32_t t1 = static_cast<uint32_t>(uint64_t(T) * (blockIdx.x + 1) / gridDim.x);
    const uint32_t tid = threadIdx.x;
    uint32_t curNode = 0xFFFFFFFFu;
    auto flush = [&]() {
        __syncthreads();
        if (curNode != 0xFFFFFFFFu) {
            for (uint32_t i = tid; i < kMaxBranch * kDims; i += blockDim.x) {
                const uint32_t v = acc[i / kDims][i % kDims];
                if (v) atomicAdd(lv.sums + uint64_t(curNode) * kMaxBranch * kDims + i, (unsigned long long)v);
            }
            if (tid < kMaxBranch && cnt[tid]) atomicAdd(lv.counts + uint64_t(curNode) * kMaxBranch + tid, cnt[tid]);
            if (tid == 0 && chg) atomicAdd(lv.changed + curNode, chg);
        }
        __syncthreads();
    };
    for (uint32_t t = t0; t < t1; t++) {
        const NodeTile ti = tiles[t];
        if (lv.lastChanged[ti.node] == 0) continue; // frozen node (kmeans.cu:238-240)
        if (ti.node != curNode) {
            flush();
            curNode = ti.node;
            for (uint32_t i = tid; i < kMaxBranch * 8; i += blockDim.x)
                (&cs[0][0])[i] = reinterpret_cast<const uint4*>(lv.centers + uint64_t(curNode) * kMaxBranch * kDims)[i];
            if (tid < kMaxBranch) {
                cn[tid] = lv.cnorm[uint64_t(curNode) * kMaxBranch + tid];
                cnt[tid] = 0;
            }
            for (uint32_t i = tid; i < kMaxBranch * (kDims + 4); i += blockDim.x) (&acc[0][0])[i] = 0;
            if (tid == 0) chg = 0;
            __syncthreads();
        }
        if (tid < ti.count) {
            const uint64_t at = uint64_t(ti.start) + tid;
            const uint32_t d = lv.members[at];
            uint4 x[8];
            const uint4* xs = reinterpret_cast<const uint4*>(lv.desc + uint64_t(d) * kDims);
#pragma unroll
            for (int k = 0; k < 8; k++) x[k] = __ldg(xs + k);
            int32_t best = 0;
            uint32_t bi = 0;
            for (uint32_t b = 0; b < kMaxBranch; b++) {
                uint32_t dot = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const uint4 c = cs[b][k];
                    dot = __dp4a(x[k].x, c.x, dot);
                    dot = __dp4a(x[k].y, c.y, dot);
                    dot = __dp4a(x[k].z, c.z, dot);
                    dot = __dp4a(x[k].w, c.w, dot);
                }
                const int32_t s = cn[b] - 2 * static_cast<int32_t>(dot);
                if (b == 0 || s < best) {
                    best = s;
                    bi = b;
                }
            }
            const uint8_t old = lv.assign[at];
            if (old != bi) atomicAdd(&chg, 1u);
            lv.assign[at] = static_cast<uint8_t>(bi);
            atomicAdd(&cnt[bi], 1u);
            // 128 shared-memory atomics per member; rows are padded to 132 words so members of
            // different centers start on different banks.
            uint32_t* a = &acc[bi][0];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t w4[4] = {x[k].x, x[k].y, x[k].z, x[k].w};
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const uint32_t v = w4[q];
                    const int base = k * 16 + q * 4;
                    atomicAdd(a + base + 0, v & 0xFFu);
                    atomicAdd(a + base + 1, (v >> 8) & 0xFFu);
                    atomicAdd(a + base + 2, (v >> 16) & 0xFFu);
                    atomicAdd(a + base + 3, v >> 24);
                }
            }
        }
        __syncthreads();
    }
    flush();
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
    const uint32_t grid = std::max(1u, std::min<uint32_t>(maxTiles, static_cast<uint32_t>(sms) * 8));
    ScopedKernelTimer timer(kTimedAssign, s);
    assignKernel<<<grid, kAssignThreads, 0, s>>>(lv, tiles, nTilesDev);
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
