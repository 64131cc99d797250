// One rank's part of a hierarchical k-means build whose descriptors are sharded across ranks
// (GPUs).  No counterpart in the reference, which builds on one GPU (Vocabulary.cpp:32-121); the
// per-level steps are its assign / update / regroup (kmeans.cu:125-199, 356-372,
// Vocabulary.cpp:83-98) split at the one point where ranks must agree: the per-node center sums,
// counts and change counts of every Lloyd step, which the caller all-reduces between assign and
// update (the reduced values are identical on every rank, so every rank applies the same update
// and keeps the same centers).  The caller's driver (rapidbow_b200/distributed.py) also chooses
// the initial centers from the all-gathered node sizes.  Shards are contiguous ranges of the
// descriptors, and every step keeps members in descriptor order, so a node's members over all
// ranks, rank by rank, are the single-GPU build's members in the same order.
#include "capi_internal.h"
#include "kmeans.cuh"

#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

namespace rbw {
namespace {

__global__ void iotaShardKernel(uint32_t* p, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) p[i] = static_cast<uint32_t>(i);
}

// rows[i] = desc[members[nodeOff[node[i]] + pos[i]]] (pos < the node's count, checked by the host).
__global__ void memberRowsKernel(const uint8_t* desc, const uint32_t* members, const uint32_t* nodeOff,
                                 const uint32_t* node, const uint32_t* pos, uint32_t count, uint8_t* rows)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; // (row, 16-byte chunk)
    if (i >= uint64_t(count) * 8) return;
    const uint32_t r = static_cast<uint32_t>(i / 8), c = static_cast<uint32_t>(i % 8);
    const uint32_t d = members[uint64_t(nodeOff[node[r]]) + pos[r]];
    reinterpret_cast<uint4*>(rows + uint64_t(r) * kDims)[c] = reinterpret_cast<const uint4*>(desc + uint64_t(d) * kDims)[c];
}

// rows[i] = desc[idx[i]] (local descriptor indices, checked by the host).
__global__ void descRowsKernel(const uint8_t* desc, const uint32_t* idx, uint32_t count, uint8_t* rows)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= uint64_t(count) * 8) return;
    const uint32_t r = static_cast<uint32_t>(i / 8), c = static_cast<uint32_t>(i % 8);
    reinterpret_cast<uint4*>(rows + uint64_t(r) * kDims)[c] =
        reinterpret_cast<const uint4*>(desc + uint64_t(idx[r]) * kDims)[c];
}

// Centers of the nodes whose reduced change count is non-zero: round(sum / count) with the
// correctly rounded quotient (kmeans.cu:356-372 with IEEE division), kept when count = 0; and
// their |c|^2.  The reduced buffers are only read.
__global__ void __launch_bounds__(256) shardUpdateKernel(uint32_t B, const unsigned long long* sums,
                                                         const uint32_t* counts, const uint32_t* changed,
                                                         uint8_t* centers, int32_t* cnorm)
{
    const uint32_t g = blockIdx.x;
    if (changed[g] == 0) return;
    uint8_t* c = centers + uint64_t(g) * kMaxBranch * kDims;
    for (uint32_t i = threadIdx.x; i < kMaxBranch * kDims; i += blockDim.x) {
        const uint32_t b = i / kDims;
        const uint32_t n = counts[uint64_t(g) * kMaxBranch + b];
        if (b < B && n != 0) c[i] = static_cast<uint8_t>(roundf(__fdiv_rn(float(sums[uint64_t(g) * kMaxBranch * kDims + i]),
                                                                          float(n))));
    }
    __syncthreads();
    if (threadIdx.x < B) {
        const uint4* c4 = reinterpret_cast<const uint4*>(c + threadIdx.x * kDims);
        uint32_t acc = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint4 v = c4[k];
            acc = __dp4a(v.x, v.x, acc);
            acc = __dp4a(v.y, v.y, acc);
            acc = __dp4a(v.z, v.z, acc);
            acc = __dp4a(v.w, v.w, acc);
        }
        cnorm[uint64_t(g) * kMaxBranch + threadIdx.x] = static_cast<int32_t>(acc);
    }
}

uint32_t blocksOf(uint64_t n, uint32_t t) { return static_cast<uint32_t>((n + t - 1) / t); }

} // namespace

class KMeansShard
{
public:
    KMeansShard(const uint8_t* desc, uint32_t n, uint32_t B, uint32_t L, cudaStream_t s)
        : mDesc{desc}, mN{n}, mB{B}, mL{L}, mStream{s}
    {
        if (B < 2 || B > kMaxBranch) throw Error(kUnsupported, "branch factor must be in [2, 16]");
        if (L < 1 || L > 8 || ipow(B, L) > 0xFFFFFFFFull) throw Error(kUnsupported, "unsupported number of levels");
        if (n != 0 && (desc == nullptr || reinterpret_cast<uintptr_t>(desc) % 16 != 0))
            throw Error(kInvalidArg, "descriptors must be 16-byte aligned device memory");
        const uint64_t maxLevel = ipow(B, L - 1), maxChild = ipow(B, L);
        mMaxTiles128 = static_cast<uint32_t>(uint64_t(n) / 128 + maxLevel + 1);
        mMaxTiles32 = static_cast<uint32_t>(uint64_t(n) / 32 + maxLevel + 1);
        mMembers.reset(std::max<uint64_t>(n, 1) * 4);
        mMembers2.reset(std::max<uint64_t>(n, 1) * 4);
        mAssign.reset(std::max<uint64_t>(n, 1));
        mNodeCnt.reset(maxChild * 4);
        mNodeOff.reset(maxChild * 4);
        mChildCnt.reset(maxChild * 4);
        mChildOff.reset(maxChild * 4);
        mCenters.reset(maxLevel * kMaxBranch * kDims);
        mCnorm.reset(maxLevel * kMaxBranch * 4);
        mSmall.reset(64);
        mTiles128.reset(uint64_t(mMaxTiles128) * sizeof(NodeTile));
        mTiles32.reset(uint64_t(mMaxTiles32) * sizeof(NodeTile));
        mTileOff.reset(maxLevel * 4);
        mScanTmp.reset(scanTempWords(std::max<uint64_t>(uint64_t(B) * mMaxTiles32, maxLevel)) * 4);
        mTileHist.reset(uint64_t(B) * mMaxTiles32 * 4);
        mTileScan.reset(uint64_t(B) * mMaxTiles32 * 4);
        mErrors.reset(sizeof(DeviceErrors));
        RBW_CUDA(cudaMemset(mErrors.get(), 0, sizeof(DeviceErrors)));
        if (n) iotaShardKernel<<<blocksOf(n, 256), 256, 0, s>>>(mMembers.as<uint32_t>(), n);
        RBW_CUDA(cudaGetLastError());
        const uint32_t zero = 0;
        RBW_CUDA(cudaMemcpyAsync(mNodeCnt.get(), &n, 4, cudaMemcpyHostToDevice, s));
        RBW_CUDA(cudaMemcpyAsync(mNodeOff.get(), &zero, 4, cudaMemcpyHostToDevice, s));
        RBW_CUDA(cudaMemsetAsync(mAssign.get(), 0, mAssign.bytes(), s));
        RBW_CUDA(cudaStreamSynchronize(s));
    }

    uint32_t level() const { return mLevel; }
    uint32_t nodes() const { return static_cast<uint32_t>(ipow(mB, mLevel)); }

    void nodeCounts(uint32_t* host) const
    {
        RBW_CUDA(cudaMemcpyAsync(host, mNodeCnt.get(), uint64_t(nodes()) * 4, cudaMemcpyDeviceToHost, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
    }

    void memberRows(const uint32_t* node, const uint32_t* pos, uint32_t count, uint8_t* hostRows) const
    {
        if (count == 0) return;
        std::vector<uint32_t> cnt(nodes());
        nodeCounts(cnt.data());
        for (uint32_t i = 0; i < count; i++)
            if (node[i] >= nodes() || pos[i] >= cnt[node[i]]) throw Error(kInvalidArg, "member position out of range");
        DeviceBuffer dIdx(uint64_t(count) * 8), dRows(uint64_t(count) * kDims);
        RBW_CUDA(cudaMemcpy(dIdx.get(), node, uint64_t(count) * 4, cudaMemcpyHostToDevice));
        RBW_CUDA(cudaMemcpy(dIdx.as<uint32_t>() + count, pos, uint64_t(count) * 4, cudaMemcpyHostToDevice));
        memberRowsKernel<<<blocksOf(uint64_t(count) * 8, 256), 256, 0, mStream>>>(
            mDesc, mMembers.as<uint32_t>(), mNodeOff.as<uint32_t>(), dIdx.as<uint32_t>(), dIdx.as<uint32_t>() + count,
            count, dRows.as<uint8_t>());
        RBW_CUDA(cudaGetLastError());
        RBW_CUDA(cudaMemcpyAsync(hostRows, dRows.get(), uint64_t(count) * kDims, cudaMemcpyDeviceToHost, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
    }

    void descRows(const uint32_t* idx, uint32_t count, uint8_t* hostRows) const
    {
        if (count == 0) return;
        for (uint32_t i = 0; i < count; i++)
            if (idx[i] >= mN) throw Error(kInvalidArg, "descriptor index out of range");
        DeviceBuffer dIdx(uint64_t(count) * 4), dRows(uint64_t(count) * kDims);
        RBW_CUDA(cudaMemcpy(dIdx.get(), idx, uint64_t(count) * 4, cudaMemcpyHostToDevice));
        descRowsKernel<<<blocksOf(uint64_t(count) * 8, 256), 256, 0, mStream>>>(mDesc, dIdx.as<uint32_t>(), count,
                                                                                 dRows.as<uint8_t>());
        RBW_CUDA(cudaGetLastError());
        RBW_CUDA(cudaMemcpyAsync(hostRows, dRows.get(), uint64_t(count) * kDims, cudaMemcpyDeviceToHost, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
    }

    // The level's initial centers ([nodes][B][128]); builds the level's member tiles.
    void setCenters(const uint8_t* host)
    {
        const uint32_t nb = nodes();
        std::vector<uint8_t> padded(uint64_t(nb) * kMaxBranch * kDims, 0);
        for (uint32_t g = 0; g < nb; g++)
            std::memcpy(padded.data() + uint64_t(g) * kMaxBranch * kDims, host + uint64_t(g) * mB * kDims,
                        uint64_t(mB) * kDims);
        RBW_CUDA(cudaMemcpy(mCenters.get(), padded.data(), padded.size(), cudaMemcpyHostToDevice));
        KMeansLevel lv = level0();
        launchCenterNorms(lv, mStream);
        buildNodeTiles(lv.nodeCnt, lv.nodeOff, nb, 128, mTileOff.as<uint32_t>(), mScanTmp.as<uint32_t>(),
                       mTiles128.as<NodeTile>(), mMaxTiles128, mSmall.as<uint32_t>(), mStream);
        RBW_CUDA(cudaMemsetAsync(mAssign.get(), 0, mAssign.bytes(), mStream)); // fresh assignment memory
        RBW_CUDA(cudaStreamSynchronize(mStream));
        mHaveCenters = true;
    }

    // Local assign step: accumulates the local sums, counts and change counts of every node whose
    // reduced change count of the previous step (lastChanged) is non-zero into the caller's
    // device buffers ([nodes][16][128] u64, [nodes][16] u32, [nodes] u32).
    void assign(const uint32_t* lastChanged, unsigned long long* sums, uint32_t* counts, uint32_t* changed)
    {
        if (!mHaveCenters) throw Error(kInvalidArg, "set the level's centers first");
        KMeansLevel lv = level0();
        lv.lastChanged = const_cast<uint32_t*>(lastChanged);
        lv.sums = sums;
        lv.counts = counts;
        lv.changed = changed;
        launchAssign(lv, mTiles128.as<NodeTile>(), mSmall.as<uint32_t>(), mMaxTiles128, mStream);
    }

    // Update from the reduced (all-rank) sums, counts and change counts.
    void update(const unsigned long long* sums, const uint32_t* counts, const uint32_t* changed)
    {
        if (!mHaveCenters) throw Error(kInvalidArg, "set the level's centers first");
        shardUpdateKernel<<<nodes(), 256, 0, mStream>>>(mB, sums, counts, changed, mCenters.as<uint8_t>(),
                                                        mCnorm.as<int32_t>());
        RBW_CUDA(cudaGetLastError());
    }

    void getCenters(uint8_t* host) const
    {
        const uint32_t nb = nodes();
        std::vector<uint8_t> padded(uint64_t(nb) * kMaxBranch * kDims);
        RBW_CUDA(cudaMemcpyAsync(padded.data(), mCenters.get(), padded.size(), cudaMemcpyDeviceToHost, mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
        for (uint32_t g = 0; g < nb; g++)
            std::memcpy(host + uint64_t(g) * mB * kDims, padded.data() + uint64_t(g) * kMaxBranch * kDims,
                        uint64_t(mB) * kDims);
    }

    // Stable regroup of the local members into the next level's nodes; writes the local child
    // counts ([nodes][B]) when hostChild is not null.
    void nextLevel(uint32_t* hostChild)
    {
        if (!mHaveCenters) throw Error(kInvalidArg, "set the level's centers first");
        if (mLevel >= mL) throw Error(kInvalidArg, "all levels are done");
        KMeansLevel lv = level0();
        RegroupScratch rs{mTileHist.as<uint32_t>(), mTileScan.as<uint32_t>(), mScanTmp.as<uint32_t>(),
                          mTiles32.as<NodeTile>(), mTileOff.as<uint32_t>(), mSmall.as<uint32_t>(), mMaxTiles32};
        launchRegroup(lv, rs, mMembers2.as<uint32_t>(), mChildCnt.as<uint32_t>(), mChildOff.as<uint32_t>(), mStream);
        if (hostChild)
            RBW_CUDA(cudaMemcpyAsync(hostChild, mChildCnt.get(), uint64_t(nodes()) * mB * 4, cudaMemcpyDeviceToHost,
                                     mStream));
        RBW_CUDA(cudaStreamSynchronize(mStream));
        std::swap(mMembers, mMembers2);
        std::swap(mNodeCnt, mChildCnt);
        std::swap(mNodeOff, mChildOff);
        mLevel++;
        mHaveCenters = false;
        const DeviceErrors e = takeErrors();
        if (e.code != 0) throw Error(kTimeout, "a bounded device wait gave up (site " + std::to_string(e.where) + ")");
    }

private:
    KMeansLevel level0() const
    {
        KMeansLevel lv{};
        lv.B = mB;
        lv.nbNodes = nodes();
        lv.nbMembers = mN;
        lv.desc = mDesc;
        lv.members = mMembers.as<uint32_t>();
        lv.nodeOff = mNodeOff.as<uint32_t>();
        lv.nodeCnt = mNodeCnt.as<uint32_t>();
        lv.centers = mCenters.as<uint8_t>();
        lv.cnorm = mCnorm.as<int32_t>();
        lv.assign = mAssign.as<uint8_t>();
        lv.ieeeDivision = 1;
        lv.err = mErrors.as<DeviceErrors>();
        return lv;
    }
    DeviceErrors takeErrors() const
    {
        DeviceErrors e{};
        RBW_CUDA(cudaMemcpy(&e, mErrors.get(), sizeof(e), cudaMemcpyDeviceToHost));
        RBW_CUDA(cudaMemset(mErrors.get(), 0, sizeof(e)));
        return e;
    }

    const uint8_t* mDesc;
    uint32_t mN, mB, mL;
    cudaStream_t mStream;
    uint32_t mLevel = 0;
    bool mHaveCenters = false;
    uint32_t mMaxTiles128 = 0, mMaxTiles32 = 0;
    DeviceBuffer mMembers, mMembers2, mAssign, mNodeCnt, mNodeOff, mChildCnt, mChildOff, mCenters, mCnorm, mSmall;
    DeviceBuffer mTiles128, mTiles32, mTileOff, mScanTmp, mTileHist, mTileScan, mErrors;
};

} // namespace rbw

struct rbw_kmeans_shard {
    std::unique_ptr<rbw::KMeansShard> s;
};
struct rbw_init_picker {
    std::mt19937_64 rng{}; // kmeans.cpp:145 (default seed, one engine per build)
};

namespace {
rbw::KMeansShard& shardOf(rbw_kmeans_shard* h)
{
    if (h == nullptr || !h->s) throw rbw::Error(rbw::kInvalidArg, "null shard handle");
    return *h->s;
}
} // namespace

extern "C" {

int rbw_kmeans_shard_create(const void* dev_desc, uint32_t nb_desc, uint32_t branch_factor, uint32_t nb_levels,
                            void* stream, rbw_kmeans_shard** out)
{
    return rbw::runGuarded([&] {
        if (out == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output handle");
        *out = nullptr;
        auto s = std::make_unique<rbw::KMeansShard>(static_cast<const uint8_t*>(dev_desc), nb_desc, branch_factor,
                                                    nb_levels, static_cast<cudaStream_t>(stream));
        *out = new rbw_kmeans_shard{std::move(s)};
    });
}

void rbw_kmeans_shard_destroy(rbw_kmeans_shard* h) { delete h; }

int rbw_kmeans_shard_level(rbw_kmeans_shard* h, uint32_t* level, uint32_t* nb_nodes)
{
    return rbw::runGuarded([&] {
        auto& s = shardOf(h);
        if (level) *level = s.level();
        if (nb_nodes) *nb_nodes = s.nodes();
    });
}

int rbw_kmeans_shard_node_counts(rbw_kmeans_shard* h, uint32_t* host_counts)
{
    return rbw::runGuarded([&] {
        if (host_counts == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        shardOf(h).nodeCounts(host_counts);
    });
}

int rbw_kmeans_shard_member_rows(rbw_kmeans_shard* h, const uint32_t* host_node, const uint32_t* host_pos,
                                 uint32_t count, uint8_t* host_rows)
{
    return rbw::runGuarded([&] {
        if (count && (host_node == nullptr || host_pos == nullptr || host_rows == nullptr))
            throw rbw::Error(rbw::kInvalidArg, "null argument");
        shardOf(h).memberRows(host_node, host_pos, count, host_rows);
    });
}

int rbw_kmeans_shard_desc_rows(rbw_kmeans_shard* h, const uint32_t* host_idx, uint32_t count, uint8_t* host_rows)
{
    return rbw::runGuarded([&] {
        if (count && (host_idx == nullptr || host_rows == nullptr)) throw rbw::Error(rbw::kInvalidArg, "null argument");
        shardOf(h).descRows(host_idx, count, host_rows);
    });
}

int rbw_kmeans_shard_set_centers(rbw_kmeans_shard* h, const uint8_t* host_centers)
{
    return rbw::runGuarded([&] {
        if (host_centers == nullptr) throw rbw::Error(rbw::kInvalidArg, "null argument");
        shardOf(h).setCenters(host_centers);
    });
}

int rbw_kmeans_shard_assign(rbw_kmeans_shard* h, const uint32_t* dev_last_changed, uint64_t* dev_sums,
                            uint32_t* dev_counts, uint32_t* dev_changed)
{
    return rbw::runGuarded([&] {
        if (!dev_last_changed || !dev_sums || !dev_counts || !dev_changed)
            throw rbw::Error(rbw::kInvalidArg, "null argument");
        shardOf(h).assign(dev_last_changed, reinterpret_cast<unsigned long long*>(dev_sums), dev_counts, dev_changed);
    });
}

int rbw_kmeans_shard_update(rbw_kmeans_shard* h, const uint64_t* dev_sums, const uint32_t* dev_counts,
                            const uint32_t* dev_changed)
{
    return rbw::runGuarded([&] {
        if (!dev_sums || !dev_counts || !dev_changed) throw rbw::Error(rbw::kInvalidArg, "null argument");
        shardOf(h).update(reinterpret_cast<const unsigned long long*>(dev_sums), dev_counts, dev_changed);
    });
}

int rbw_kmeans_shard_get_centers(rbw_kmeans_shard* h, uint8_t* host_centers)
{
    return rbw::runGuarded([&] {
        if (host_centers == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        shardOf(h).getCenters(host_centers);
    });
}

int rbw_kmeans_shard_next_level(rbw_kmeans_shard* h, uint32_t* host_child_counts)
{
    return rbw::runGuarded([&] { shardOf(h).nextLevel(host_child_counts); });
}

int rbw_init_picker_create(rbw_init_picker** out)
{
    return rbw::runGuarded([&] {
        if (out == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output handle");
        *out = new rbw_init_picker{};
    });
}

void rbw_init_picker_destroy(rbw_init_picker* p) { delete p; }

int rbw_init_picker_level(rbw_init_picker* p, uint32_t branch_factor, const uint32_t* node_counts, uint32_t nb_nodes,
                          uint32_t* positions, uint32_t* n_valid)
{
    return rbw::runGuarded([&] {
        if (p == nullptr || (nb_nodes && (node_counts == nullptr || positions == nullptr || n_valid == nullptr)))
            throw rbw::Error(rbw::kInvalidArg, "null argument");
        if (branch_factor < 2 || branch_factor > rbw::kMaxBranch) throw rbw::Error(rbw::kInvalidArg, "bad branch factor");
        for (uint32_t g = 0; g < nb_nodes; g++)
            n_valid[g] = rbw::referencePick(p->rng, positions + uint64_t(g) * branch_factor, node_counts[g],
                                            branch_factor);
    });
}

int rbw_idf_weights(uint32_t nb_doc, const uint32_t* occ, uint64_t n, float* weights)
{
    return rbw::runGuarded([&] {
        if (n && (occ == nullptr || weights == nullptr)) throw rbw::Error(rbw::kInvalidArg, "null argument");
        for (uint64_t i = 0; i < n; i++) weights[i] = rbw::idfWeight(nb_doc, occ[i]);
    });
}

} // extern "C"
