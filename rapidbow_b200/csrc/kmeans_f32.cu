// Float-center k-means and lookup.  No counterpart in the reference, whose centers are uint8
// (kmeans.cu:367); this mode generalises its assign and update (kmeans.cu:125-199, 356-372):
//
//   * centers are fp32: c = float(double(sum) / double(count)) from the exact integer sums,
//     kept when a center has no member (kmeans.cu:360-362);
//   * distances: score_b = |c_b|^2 - 2 x.c_b with x.c_b from the tensor core.  x (uint8) is
//     exact in bf16; every center is split into hi = bf16(c) and lo = bf16(c - hi), and one
//     tcgen05.mma.kind::f16 (M = 128 members, N = 32 = 16 hi + 16 lo rows, fp32 accumulation)
//     gives x.hi and x.lo, added in fp32;
//   * error bound: |score error| <= 4e-5 (|x||c| + |c|^2) (the split leaves |c - hi - lo| <=
//     2^-18 |c|; the products are exact in fp32; at most 127 accumulation roundings of <= 2^-23
//     each; |c|^2 and the final subtraction round once more), so a member whose best-versus-
//     second margin is at most kMarginScale (|x| max|c| + max|c|^2) -- six times the bound for
//     both scores together -- is re-scored in FP64: the warp computes its squared distance to
//     every center in the oracle's fixed order (lane partials of four fused multiply-adds, then
//     a butterfly of pairwise sums) and keeps the lowest index on ties (kmeans.cu:131-135);
//     every other member's fp32 argmin is the FP64 argmin by a margin;
//   * inertia: per node, sum_b (Q_b - 2 c_b.S_b + n_b |c_b|^2) in FP64 from the exact member
//     sums S_b, counts n_b and sums of squared norms Q_b, with the centers of the assignment.
#include "kmeans.cuh"
#include "timing.h"
#include "tuning.h"

#include <cuda_bf16.h>

#include <algorithm>

namespace rbw {
namespace {

constexpr float kMarginScale = 1.0f / 2048.0f;

__device__ __forceinline__ uint32_t packBf16x2(float a, float b)
{
    const __nv_bfloat16 ha = __float2bfloat16_rn(a), hb = __float2bfloat16_rn(b);
    return uint32_t(__bfloat16_as_ushort(ha)) | (uint32_t(__bfloat16_as_ushort(hb)) << 16);
}

// hi and lo bf16 parts of two values, packed as bf16x2 (first value in the low half).
__device__ __forceinline__ void splitPair(float a, float b, uint32_t& hi, uint32_t& lo)
{
    const __nv_bfloat16 ha = __float2bfloat16_rn(a), hb = __float2bfloat16_rn(b);
    hi = uint32_t(__bfloat16_as_ushort(ha)) | (uint32_t(__bfloat16_as_ushort(hb)) << 16);
    lo = packBf16x2(a - __bfloat162float(ha), b - __bfloat162float(hb));
}

// Split, |c|^2 and bound of one node (256 threads: thread t handles dims 8 (t % 16) .. +7 of
// center t / 16).  `red` is 16 floats of shared memory.
__device__ void prepareNode(const float* __restrict__ c, uint8_t* __restrict__ split, float* __restrict__ cn,
                            float2* __restrict__ bound, uint32_t B, float* red)
{
    const uint32_t t = threadIdx.x;
    const uint32_t j = t / 16, part = t % 16, d0 = part * 8;
    uint32_t hi[4], lo[4];
    double nrm = 0.0;
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) {
        const float a = j < B ? c[j * kDims + d0 + 2 * k] : 0.f;
        const float b = j < B ? c[j * kDims + d0 + 2 * k + 1] : 0.f;
        splitPair(a, b, hi[k], lo[k]);
        nrm = __fma_rn(double(a), double(a), nrm);
        nrm = __fma_rn(double(b), double(b), nrm);
    }
    const uint32_t kb = d0 / 64, ch = (d0 % 64) / 8;
    uint8_t* base = split + kb * 4096;
    *reinterpret_cast<uint4*>(base + j * 128 + ((ch ^ (j & 7u)) << 4)) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    const uint32_t r = 16 + j;
    *reinterpret_cast<uint4*>(base + r * 128 + ((ch ^ (r & 7u)) << 4)) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
#pragma unroll
    for (uint32_t off = 8; off > 0; off >>= 1) nrm = __dadd_rn(nrm, __shfl_xor_sync(0xFFFFFFFFu, nrm, off));
    if (part == 0) {
        cn[j] = j < B ? __double2float_rn(nrm) : kPadNormF;
        red[j] = j < B ? __double2float_ru(nrm) : 0.f;
    }
    __syncthreads();
    if (t == 0) {
        float c2 = 0.f;
        for (uint32_t b = 0; b < B; b++) c2 = fmaxf(c2, red[b]);
        *bound = make_float2(__fsqrt_ru(c2), c2);
    }
}

__global__ void __launch_bounds__(256) centersToFloatKernel(KMeansLevelF lv)
{
    __shared__ float red[kMaxBranch];
    const uint32_t g = blockIdx.x;
    const uint8_t* u = lv.base.centers + uint64_t(g) * kMaxBranch * kDims;
    float* c = lv.centers + uint64_t(g) * kMaxBranch * kDims;
    for (uint32_t i = threadIdx.x; i < kMaxBranch * kDims; i += blockDim.x)
        c[i] = i / kDims < lv.base.B ? float(u[i]) : 0.f;
    __syncthreads();
    prepareNode(c, lv.split + uint64_t(g) * kSplitBytes, lv.cn + uint64_t(g) * kMaxBranch, lv.bound + g, lv.base.B,
                red);
}

__global__ void __launch_bounds__(256) prepareNodesKernel(const float* centers, uint8_t* split, float* cn,
                                                          float2* bound, uint32_t B)
{
    __shared__ float red[kMaxBranch];
    const uint64_t g = blockIdx.x;
    prepareNode(centers + g * kMaxBranch * kDims, split + g * kSplitBytes, cn + g * kMaxBranch, bound + g, B, red);
}

// ------------------------------------------------------------------ assign
constexpr uint32_t kAfThreads = 128;
constexpr uint32_t kAfRows = 128;
constexpr uint32_t kAfTmemCols = 32;
constexpr uint32_t kAfCtasPerSm = 3;
constexpr uint32_t kAfTileWindow = kAfThreads; // one tile entry per thread per refill
constexpr uint32_t kAfFrozen = 0x80000000u;

struct AssignFSmem {
    uint8_t a[2][kAfRows * 128];     // members as bf16, two K-blocks of 64 dims, 128-byte swizzle
    uint8_t b[2][32 * 128];          // the node's hi (rows 0-15) and lo (rows 16-31) centers
    uint8_t x8[kAfRows * kDims];     // members as uint8, row-major (sums and FP64 re-score)
    NodeTile win[kAfTileWindow];     // tiles [winBase, winBase + kAfTileWindow) of the CTA's range,
                                     // count | kAfFrozen for a frozen node
    uint32_t acc[kMaxBranch * kDims]; // center sums of the current node (accIndex layout)
    unsigned long long q[kMaxBranch];
    float cn[kMaxBranch];
    uint32_t xn[kAfRows];
    uint32_t cnt[kMaxBranch];
    uint8_t bsel[kAfRows];
    float2 bnd;
    uint64_t mmaBar;
    uint32_t tmemBase;
    uint32_t chg;
    uint32_t abortFlag;
    uint32_t refined;
    uint32_t visited;
};
constexpr size_t kAfSmemBytes = sizeof(AssignFSmem) + 1024;

__device__ __forceinline__ uint32_t accIndexF(uint32_t b, uint32_t d)
{
    return b * kDims + (d & 3u) * 32u + (d >> 2);
}

// bf16 of the four bytes of w (exact: integers below 256), packed in two bf16x2 words.
__device__ __forceinline__ void bytesToBf16(uint32_t w, uint32_t& lo2, uint32_t& hi2)
{
    const float f0 = __int_as_float(int(__byte_perm(w, 0x4B000000u, 0x7540u))) - 8388608.0f;
    const float f1 = __int_as_float(int(__byte_perm(w, 0x4B000000u, 0x7541u))) - 8388608.0f;
    const float f2 = __int_as_float(int(__byte_perm(w, 0x4B000000u, 0x7542u))) - 8388608.0f;
    const float f3 = __int_as_float(int(__byte_perm(w, 0x4B000000u, 0x7543u))) - 8388608.0f;
    // the low 16 bits of these floats are zero, so the bf16 bits are the high halves
    lo2 = (__float_as_uint(f0) >> 16) | (__float_as_uint(f1) & 0xFFFF0000u);
    hi2 = (__float_as_uint(f2) >> 16) | (__float_as_uint(f3) & 0xFFFF0000u);
}

__global__ void __launch_bounds__(kAfThreads, kAfCtasPerSm) assignKernelF(KMeansLevelF lv, const NodeTile* tiles,
                                                                         const uint32_t* nTilesDev)
{
    extern __shared__ uint8_t smemRaw[];
    AssignFSmem& S = *reinterpret_cast<AssignFSmem*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    const KMeansLevel& L0 = lv.base;
    const uint32_t tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
    const uint32_t B = L0.B;
    const bool build = lv.lookupOnly == 0;
    const uint32_t T = *nTilesDev;
    const uint32_t t0 = static_cast<uint32_t>(uint64_t(T) * blockIdx.x / gridDim.x);
    const uint32_t t1 = static_cast<uint32_t>(uint64_t(T) * (blockIdx.x + 1) / gridDim.x);
    volatile uint32_t* abortFlag = &S.abortFlag;
    if (tid == 0) {
        mbarInit(&S.mmaBar, 1);
        S.abortFlag = 0;
        S.refined = 0;
        S.visited = 0;
        fenceMbarInit();
    }
    if (warp == 0) {
        tmemAlloc(&S.tmemBase, kAfTmemCols);
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
        if (curNode != 0xFFFFFFFFu && build) {
            // plain stores for a node no other CTA touches (its accumulators are zero on entry)
            for (uint32_t i = tid; i < kMaxBranch * kDims; i += kAfThreads) {
                const uint32_t b = i / kDims, d = i % kDims;
                const uint32_t v = S.acc[accIndexF(b, d)];
                unsigned long long* dst = L0.sums + (uint64_t(curNode) * kMaxBranch + b) * kDims + d;
                if (v) {
                    if (curExclusive) *dst = v;
                    else atomicAdd(dst, (unsigned long long)v);
                }
            }
            if (tid < kMaxBranch && S.cnt[tid]) {
                uint32_t* c = L0.counts + uint64_t(curNode) * kMaxBranch + tid;
                unsigned long long* qd = lv.q + uint64_t(curNode) * kMaxBranch + tid;
                if (curExclusive) {
                    *c = S.cnt[tid];
                    *qd = S.q[tid];
                } else {
                    atomicAdd(c, S.cnt[tid]);
                    atomicAdd(qd, S.q[tid]);
                }
            }
            if (tid == 0 && S.chg) {
                if (curExclusive) L0.changed[curNode] = S.chg;
                else atomicAdd(L0.changed + curNode, S.chg);
            }
        }
        __syncthreads();
    };
    // The tile list and the frozen flags are read a window of kAfTileWindow tiles at a time (one
    // load per thread, all in flight together), the member indices two tiles ahead and the member
    // rows one tile ahead of their use, into registers, so that no tile waits on a chain of
    // dependent global loads.  Every thread runs the same window refills (uniform).
    uint32_t winBase = t0;
    auto refill = [&](uint32_t base) {
        __syncthreads(); // nobody reads the old window any more
        if (base + tid < t1) {
            NodeTile x = tiles[base + tid];
            if (build && L0.lastChanged[x.node] == 0) x.count |= kAfFrozen; // frozen node (kmeans.cu:238-240)
            S.win[tid] = x;
        }
        winBase = base;
        __syncthreads();
    };
    auto entry = [&](uint32_t t) -> NodeTile {
        if (t - winBase >= kAfTileWindow) refill(t);
        return S.win[t - winBase];
    };
    auto nextLive = [&](uint32_t t) -> uint32_t {
        for (; t < t1; t++)
            if (!(entry(t).count & kAfFrozen)) return t;
        return t1;
    };
    // rows past a tile's count repeat its first member (their results are not used)
    auto loadIndices = [&](const NodeTile& tn, uint32_t (&m)[kAfRows / 16]) {
#pragma unroll
        for (uint32_t k = 0; k < kAfRows / 16; k++) {
            const uint32_t row = 16u * k + tid / 8;
            m[k] = L0.members[uint64_t(tn.start) + (row < tn.count ? row : 0u)];
        }
    };
    const uint32_t c8 = tid % 8;
    auto loadRows = [&](const uint32_t (&m)[kAfRows / 16], uint4 (&v)[kAfRows / 16]) {
#pragma unroll
        for (uint32_t k = 0; k < kAfRows / 16; k++)
            v[k] = __ldg(reinterpret_cast<const uint4*>(L0.desc + uint64_t(m[k]) * kDims) + c8);
    };
    if (t0 < t1) refill(t0);
    uint32_t t = nextLive(t0);
    NodeTile ti{}, tn1{};
    uint32_t mNext[kAfRows / 16];
    uint4 v[kAfRows / 16];
    if (t < t1) {
        ti = entry(t);
        loadIndices(ti, mNext);
        loadRows(mNext, v);
    }
    uint32_t n1 = t < t1 ? nextLive(t + 1) : t1;
    if (n1 < t1) {
        tn1 = entry(n1);
        loadIndices(tn1, mNext);
    }
    while (t < t1) {
        if (tid == 0) S.visited += ti.count;
        if (ti.node != curNode) {
            flush();
            curNode = ti.node;
            curExclusive = ti.first >= t0 && uint64_t(ti.first) + (L0.nodeCnt[curNode] + kAfRows - 1) / kAfRows <= t1;
            const uint4* src = reinterpret_cast<const uint4*>(lv.split + uint64_t(curNode) * kSplitBytes);
#pragma unroll
            for (uint32_t k = 0; k < kSplitBytes / 16 / kAfThreads; k++)
                reinterpret_cast<uint4*>(&S.b[0][0])[tid + kAfThreads * k] = src[tid + kAfThreads * k];
            if (tid < kMaxBranch) {
                S.cn[tid] = lv.cn[uint64_t(curNode) * kMaxBranch + tid];
                S.cnt[tid] = 0;
                S.q[tid] = 0;
            }
            if (tid == 0) {
                S.bnd = lv.bound[curNode];
                S.chg = 0;
            }
            if (build)
                for (uint32_t i = tid; i < kMaxBranch * kDims; i += kAfThreads) S.acc[i] = 0;
        }
        {
            // Eight threads per row, 16 rows per round: thread c8 = tid % 8 stages dims
            // 16 c8 .. 16 c8 + 15 of its row as uint8 and as bf16 (K-block c8 / 4, 16-byte chunks
            // 2 (c8 % 4) and 2 (c8 % 4) + 1 of the 128-byte row, swizzled by the row's low bits),
            // and the eight threads add up the row's |x|^2.
#pragma unroll
            for (uint32_t k = 0; k < kAfRows / 16; k++) {
                const uint32_t row = 16u * k + tid / 8;
                *reinterpret_cast<uint4*>(S.x8 + row * kDims + c8 * 16) = v[k];
                uint32_t w[8];
                bytesToBf16(v[k].x, w[0], w[1]);
                bytesToBf16(v[k].y, w[2], w[3]);
                bytesToBf16(v[k].z, w[4], w[5]);
                bytesToBf16(v[k].w, w[6], w[7]);
                uint8_t* rowBase = S.a[c8 / 4] + row * 128;
                const uint32_t j0 = (c8 % 4) * 2;
                *reinterpret_cast<uint4*>(rowBase + ((j0 ^ (row & 7u)) << 4)) = make_uint4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<uint4*>(rowBase + (((j0 + 1) ^ (row & 7u)) << 4)) = make_uint4(w[4], w[5], w[6], w[7]);
                uint32_t xn = __dp4a(v[k].x, v[k].x, 0u);
                xn = __dp4a(v[k].y, v[k].y, xn);
                xn = __dp4a(v[k].z, v[k].z, xn);
                xn = __dp4a(v[k].w, v[k].w, xn);
                xn += __shfl_xor_sync(0xFFFFFFFFu, xn, 1);
                xn += __shfl_xor_sync(0xFFFFFFFFu, xn, 2);
                xn += __shfl_xor_sync(0xFFFFFFFFu, xn, 4);
                if (c8 == 0) S.xn[row] = xn;
            }
        }
        // the next live tile's rows into registers (its indices were loaded one tile ago), the
        // indices of the one after it; both land while this tile is scored
        uint32_t n2 = t1;
        NodeTile tn2{};
        if (n1 < t1) {
            loadRows(mNext, v);
            n2 = nextLive(n1 + 1);
            if (n2 < t1) {
                tn2 = entry(n2);
                loadIndices(tn2, mNext);
            }
        }
        const uint32_t row = tid;
        const bool valid = row < ti.count;
        const uint64_t at = uint64_t(ti.start) + row;
        const uint32_t prevAssign = build && valid ? L0.assign[at] : 0u; // lands during the MMA
        // generic-proxy shared-memory writes read by the tensor core
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tcFenceAfter();
            const uint32_t aBase = smemAddr(&S.a[0][0]), bBase = smemAddr(&S.b[0][0]);
#pragma unroll
            for (uint32_t k = 0; k < 8; k++) {
                mmaBf16(tmem, smemDescSw128(aBase + (k >> 2) * (kAfRows * 128) + 32u * (k & 3u)),
                        smemDescSw128(bBase + (k >> 2) * (32 * 128) + 32u * (k & 3u)), idescBf16(32), k > 0 ? 1u : 0u);
            }
            mmaCommit(&S.mmaBar);
        }
        if (!mbarWait(&S.mmaBar, phase, abortFlag, L0.err, 50)) break;
        phase ^= 1u;
        tcFenceAfter();
        uint32_t rh[16], rl[16];
        tmemLoad16(tmem + ((warp * 32u) << 16), rh);
        tmemLoad16(tmem + ((warp * 32u) << 16) + 16u, rl);
        tmemWaitTie(rh);
        tmemWaitTie(rl);
        tcFenceBefore(); // the next tile's MMA overwrites these columns after the barriers below
        float best = __int_as_float(0x7F800000), second = best;
        uint32_t bi = 0;
#pragma unroll
        for (uint32_t b = 0; b < kMaxBranch; b++) {
            if (b < B) {
                const float dot = __fadd_rn(__uint_as_float(rh[b]), __uint_as_float(rl[b]));
                const float s = __fmaf_rn(-2.f, dot, S.cn[b]);
                if (s < best) {
                    second = best;
                    best = s;
                    bi = b;
                } else if (s < second) {
                    second = s;
                }
            }
        }
        const float thr = kMarginScale * __fmaf_rn(__fsqrt_ru(float(S.xn[row])), S.bnd.x, S.bnd.y);
        const bool refine = valid && !(second - best > thr);
        uint32_t mask = __ballot_sync(0xFFFFFFFFu, refine);
        if (mask != 0) {
            // FP64 re-score of the flagged rows of this warp, one row at a time, every lane on
            // dims 4 lane .. 4 lane + 3 of every center (the oracle's orc_dist64 order).
            if (lane == 0) atomicAdd(&S.refined, uint32_t(__popc(mask)));
            const float* cBase = lv.centers + uint64_t(curNode) * kMaxBranch * kDims + 4u * lane;
            while (mask != 0) {
                const uint32_t src = __ffs(mask) - 1;
                mask &= mask - 1;
                const uint32_t xw = *reinterpret_cast<const uint32_t*>(S.x8 + (warp * 32u + src) * kDims + 4u * lane);
                double bestD = 0.0;
                uint32_t bb = 0;
                for (uint32_t b = 0; b < B; b++) {
                    const float4 c4 = __ldg(reinterpret_cast<const float4*>(cBase + b * kDims));
                    double p = 0.0;
                    double e = __dsub_rn(double(xw & 0xFFu), double(c4.x));
                    p = __fma_rn(e, e, p);
                    e = __dsub_rn(double((xw >> 8) & 0xFFu), double(c4.y));
                    p = __fma_rn(e, e, p);
                    e = __dsub_rn(double((xw >> 16) & 0xFFu), double(c4.z));
                    p = __fma_rn(e, e, p);
                    e = __dsub_rn(double(xw >> 24), double(c4.w));
                    p = __fma_rn(e, e, p);
#pragma unroll
                    for (uint32_t off = 16; off > 0; off >>= 1) p = __dadd_rn(p, __shfl_xor_sync(0xFFFFFFFFu, p, off));
                    if (b == 0 || p < bestD) {
                        bestD = p;
                        bb = b;
                    }
                }
                if (lane == src) bi = bb;
            }
        }
        if (!build) {
            if (valid) L0.assign[uint64_t(ti.start) + row] = static_cast<uint8_t>(bi);
        } else {
            if (valid) {
                if (prevAssign != bi) atomicAdd(&S.chg, 1u);
                L0.assign[at] = static_cast<uint8_t>(bi);
                atomicAdd(&S.cnt[bi], 1u);
                atomicAdd(&S.q[bi], (unsigned long long)S.xn[row]);
            }
            S.bsel[row] = static_cast<uint8_t>(bi);
            __syncwarp();
            const uint32_t rEnd = ti.count < 32u * warp + 32u ? ti.count : 32u * warp + 32u;
            for (uint32_t rr = 32u * warp; rr < rEnd; rr++) {
                const uint32_t b = S.bsel[rr];
                const uint32_t x = *reinterpret_cast<const uint32_t*>(S.x8 + rr * kDims + 4u * lane);
                uint32_t* a = S.acc + b * kDims + lane;
                atomicAdd(a, x & 0xFFu);
                atomicAdd(a + 32, (x >> 8) & 0xFFu);
                atomicAdd(a + 64, (x >> 16) & 0xFFu);
                atomicAdd(a + 96, x >> 24);
            }
        }
        __syncthreads(); // the tiles, bsel and xn are rewritten by the next step
        t = n1;
        ti = tn1;
        n1 = n2;
        tn1 = tn2;
    }
    flush();
    if (tid == 0) {
        if (S.refined) atomicAdd(lv.refined, (unsigned long long)S.refined);
        if (S.visited) atomicAdd(lv.refined + 1, (unsigned long long)S.visited);
    }
    if (warp == 0) {
        tcFenceAfter();
        tmemDealloc(tmem, kAfTmemCols);
    }
}

// ------------------------------------------------------------------ update
__global__ void __launch_bounds__(256) updateKernelF(KMeansLevelF lv)
{
    __shared__ uint32_t ch, ran;
    __shared__ uint32_t cnt[kMaxBranch];
    __shared__ double term[kMaxBranch];
    __shared__ float red[kMaxBranch];
    const KMeansLevel& L0 = lv.base;
    const uint32_t g = blockIdx.x, t = threadIdx.x, B = L0.B;
    if (t == 0) {
        const uint32_t prev = L0.lastChanged[g];
        ch = L0.changed[g];
        ran = prev != 0 ? 1u : 0u; // the assign step visited this node
        L0.lastChanged[g] = ch;
        L0.changed[g] = 0;
        if (ch != 0) atomicAdd(L0.activeCount, 1u);
    }
    if (t < kMaxBranch) cnt[t] = L0.counts[uint64_t(g) * kMaxBranch + t];
    __syncthreads();
    // A node frozen before this step was skipped by the assign (ch is 0 then): nothing was
    // accumulated, every counter is zero and its inertia is that of its last assignment.
    if (!ran) return;
    float* c = lv.centers + uint64_t(g) * kMaxBranch * kDims;
    unsigned long long* sums = L0.sums + uint64_t(g) * kMaxBranch * kDims;
    unsigned long long* q = lv.q + uint64_t(g) * kMaxBranch;
    if (ran) {
        // inertia of the assignment just made, with the centers it was made against
        const uint32_t j = t / 16, part = t % 16;
        double cs = 0.0, cc = 0.0;
#pragma unroll
        for (uint32_t k = 0; k < 8; k++) {
            const uint32_t d = part * 8 + k;
            const double cv = double(c[j * kDims + d]);
            cs = __fma_rn(cv, double(sums[j * kDims + d]), cs);
            cc = __fma_rn(cv, cv, cc);
        }
#pragma unroll
        for (uint32_t off = 8; off > 0; off >>= 1) {
            cs = __dadd_rn(cs, __shfl_xor_sync(0xFFFFFFFFu, cs, off));
            cc = __dadd_rn(cc, __shfl_xor_sync(0xFFFFFFFFu, cc, off));
        }
        if (part == 0)
            term[j] = j < B ? __fma_rn(double(cnt[j]), cc, __fma_rn(-2.0, cs, double(q[j]))) : 0.0;
        __syncthreads();
        if (t == 0) {
            double s = 0.0;
            for (uint32_t b = 0; b < B; b++) s = __dadd_rn(s, term[b]);
            lv.inertiaNode[g] = s;
        }
    }
    __syncthreads();
    if (ch != 0) {
        for (uint32_t i = t; i < kMaxBranch * kDims; i += blockDim.x) {
            const uint32_t b = i / kDims;
            if (b < B && cnt[b] != 0) c[i] = __double2float_rn(__ddiv_rn(double(sums[i]), double(cnt[b])));
        }
    }
    for (uint32_t i = t; i < B * kDims; i += blockDim.x) sums[i] = 0ull; // centers b >= B have none
    __syncthreads();
    if (t < B) {
        L0.counts[uint64_t(g) * kMaxBranch + t] = 0;
        q[t] = 0ull;
    }
    if (ch != 0)
        prepareNode(c, lv.split + uint64_t(g) * kSplitBytes, lv.cn + uint64_t(g) * kMaxBranch, lv.bound + g, B, red);
}

__global__ void __launch_bounds__(1024) inertiaSumKernel(const double* in, uint32_t n, double* out)
{
    __shared__ double part[1024];
    double s = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += 1024) s = __dadd_rn(s, in[i]);
    part[threadIdx.x] = s;
    __syncthreads();
    for (uint32_t off = 512; off > 0; off >>= 1) {
        if (threadIdx.x < off) part[threadIdx.x] = __dadd_rn(part[threadIdx.x], part[threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

__global__ void writeLeavesKernel(KMeansLevel lv, const NodeTile* tiles, const uint32_t* nTilesDev, uint32_t* leaf)
{
    // warp per 128-member tile
    const uint32_t T = *nTilesDev;
    const uint32_t warpsTotal = gridDim.x * (blockDim.x / 32);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t t = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; t < T; t += warpsTotal) {
        const NodeTile ti = tiles[t];
        for (uint32_t r = lane; r < ti.count; r += 32) {
            const uint64_t at = uint64_t(ti.start) + r;
            leaf[lv.members[at]] = ti.node * lv.B + lv.assign[at];
        }
    }
}

} // namespace

void launchCentersToFloat(const KMeansLevelF& lv, cudaStream_t s)
{
    if (lv.base.nbNodes == 0) return;
    centersToFloatKernel<<<lv.base.nbNodes, 256, 0, s>>>(lv);
    RBW_CUDA(cudaGetLastError());
}

void launchPrepareFloatNodes(const float* centers, uint8_t* split, float* cn, float2* bound, uint64_t nbNodes,
                             uint32_t B, cudaStream_t s)
{
    for (uint64_t off = 0; off < nbNodes; off += 0x7FFFFFFFull) {
        const uint64_t m = std::min<uint64_t>(nbNodes - off, 0x7FFFFFFFull);
        prepareNodesKernel<<<static_cast<uint32_t>(m), 256, 0, s>>>(centers + off * kMaxBranch * kDims,
                                                                     split + off * kSplitBytes, cn + off * kMaxBranch,
                                                                     bound + off, B);
        RBW_CUDA(cudaGetLastError());
    }
}

void launchAssignF(const KMeansLevelF& lv, const NodeTile* tiles, const uint32_t* nTilesDev, uint32_t maxTiles,
                   cudaStream_t s)
{
    static std::atomic<uint64_t> attrSet{0};
    setMaxDynamicSmemOncePerDevice(reinterpret_cast<const void*>(assignKernelF), static_cast<int>(kAfSmemBytes),
                                   attrSet);
    static_assert(kAfCtasPerSm * kAfTmemCols <= 512, "TMEM columns of the resident CTAs");
    static_assert(kAfCtasPerSm * kAfSmemBytes <= 227 * 1024, "shared memory of the resident CTAs");
    const uint32_t perSm =
        std::min(kAfCtasPerSm, tunedValue(kTuneAssignFCtasPerSm, lv.base.B, 0, lv.base.nbMembers));
    const uint32_t grid =
        std::max(1u, std::min<uint32_t>(maxTiles, static_cast<uint32_t>(currentSmCount()) * perSm));
    ScopedKernelTimer timer(kTimedAssign, s);
    assignKernelF<<<grid, kAfThreads, kAfSmemBytes, s>>>(lv, tiles, nTilesDev);
    RBW_CUDA(cudaGetLastError());
}

void launchUpdateF(const KMeansLevelF& lv, cudaStream_t s)
{
    if (lv.base.nbNodes == 0) return;
    ScopedKernelTimer timer(kTimedUpdate, s);
    updateKernelF<<<lv.base.nbNodes, 256, 0, s>>>(lv);
    RBW_CUDA(cudaGetLastError());
}

void launchInertiaSum(const double* inertiaNode, uint32_t nbNodes, double* out, cudaStream_t s)
{
    inertiaSumKernel<<<1, 1024, 0, s>>>(inertiaNode, nbNodes, out);
    RBW_CUDA(cudaGetLastError());
}

void launchWriteLeaves(const KMeansLevel& lv, const NodeTile* tiles, const uint32_t* nTilesDev, uint32_t maxTiles,
                       uint32_t* leaf, cudaStream_t s)
{
    const uint32_t blocks = std::max(1u, std::min<uint32_t>((maxTiles + 7) / 8, 16384));
    writeLeavesKernel<<<blocks, 256, 0, s>>>(lv, tiles, nTilesDev, leaf);
    RBW_CUDA(cudaGetLastError());
}

} // namespace rbw
