// k-means center update (kmeans.cu:334-375).  This translation unit is compiled with
// --use_fast_math, as the reference's kernels are (CMakeLists.txt:22), so the quotient
// float(sum) / float(count) below takes the same approximate-division path as kmeans.cu:367 and
// the rounded uint8 centers are bit-identical.  Sums are u64 here (u32 in the reference; equal
// whenever the reference's sum does not overflow, i.e. below 2^32).  With ieeeDivision set the
// quotient is the correctly rounded one instead (__fdiv_rn), which is what the CPU oracle computes.
#include "kmeans.cuh"
#include "timing.h"

namespace rbw {
namespace {

__global__ void __launch_bounds__(256) updateKernel(KMeansLevel lv)
{
    __shared__ uint32_t ch, frozen;
    __shared__ uint32_t cnt[kMaxBranch];
    const uint32_t g = blockIdx.x;
    if (threadIdx.x == 0) {
        ch = lv.changed[g];
        // A node frozen before this step was skipped by the assign: nothing was accumulated and
        // every counter is already zero, so there is nothing to do.
        frozen = lv.lastChanged[g] == 0 && ch == 0;
        lv.lastChanged[g] = ch;
        lv.changed[g] = 0;
        if (ch != 0) atomicAdd(lv.activeCount, 1u);
    }
    if (threadIdx.x < kMaxBranch) cnt[threadIdx.x] = lv.counts[uint64_t(g) * kMaxBranch + threadIdx.x];
    __syncthreads();
    if (frozen) return;
    // Nodes with no change keep their centers (kmeans.cu:341-343); their accumulators are still
    // cleared so the next level starts from zero.  Centers b >= B have no members: their sums
    // and counts stay zero.
    uint8_t* c = lv.centers + uint64_t(g) * kMaxBranch * kDims;
    unsigned long long* sums = lv.sums + uint64_t(g) * kMaxBranch * kDims;
    for (uint32_t i = threadIdx.x; i < lv.B * kDims; i += blockDim.x) {
        const uint32_t b = i / kDims;
        const uint32_t n = cnt[b];
        if (ch != 0 && b < lv.B && n != 0) {
            const unsigned long long s = sums[i];
            const float q = lv.ieeeDivision ? __fdiv_rn(float(s), float(n)) : float(s) / float(n);
            c[i] = static_cast<uint8_t>(roundf(q));
        }
        sums[i] = 0ull;
    }
    __syncthreads();
    if (threadIdx.x < kMaxBranch) {
        const uint32_t b = threadIdx.x;
        lv.counts[uint64_t(g) * kMaxBranch + b] = 0;
        if (ch != 0 && b < lv.B) {
            const uint4* c4 = reinterpret_cast<const uint4*>(c + b * kDims);
            uint32_t acc = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint4 v = c4[k];
                acc = __dp4a(v.x, v.x, acc);
                acc = __dp4a(v.y, v.y, acc);
                acc = __dp4a(v.z, v.z, acc);
                acc = __dp4a(v.w, v.w, acc);
            }
            lv.cnorm[uint64_t(g) * kMaxBranch + b] = static_cast<int32_t>(acc);
        }
    }
}

} // namespace

void launchUpdate(const KMeansLevel& lv, cudaStream_t s)
{
    if (lv.nbNodes == 0) return;
    ScopedKernelTimer timer(kTimedUpdate, s);
    updateKernel<<<lv.nbNodes, 256, 0, s>>>(lv);
    RBW_CUDA(cudaGetLastError());
}

} // namespace rbw
