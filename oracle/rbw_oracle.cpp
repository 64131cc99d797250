// Test infrastructure only: the oracle, a CPU restatement of the reference algorithm for the
// hot path.  It is the checker for tests/, the seed of __graft_entry__.smoke()'s check and the
// timed CPU baseline in bench.py -- never part of the product path.  Each function cites the
// reference file:line it restates.  Pinned against the reference itself (oracle/_ref, built from
// the reference sources by oracle/Makefile) by tests/test_oracle_pin*.py.
#include "rbw_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <random>
#include <thread>
#include <unordered_set>
#include <vector>

namespace {

constexpr uint32_t kDims = 128;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;

uint64_t levelBeg(uint32_t B, uint32_t level)
{
    // FullTree.h:38-52, generalised to any branching factor: 1 + B + ... + B^(level-1).
    uint64_t acc = 0;
    for (uint32_t i = 0; i < level; i++) acc = acc * B + 1;
    return acc;
}

uint64_t ipow(uint64_t b, uint32_t e)
{
    uint64_t r = 1;
    while (e--) r *= b;
    return r;
}

// Exact squared L2 distance of two 128-byte descriptors (kmeans.cuh:62-71).
inline uint32_t dist128(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b)
{
    uint32_t acc = 0;
    for (uint32_t i = 0; i < kDims; i++) {
        const int d = int(a[i]) - int(b[i]);
        acc += uint32_t(d * d);
    }
    return acc;
}

// argmin over the B centers of a node, lowest index on ties (vocTreeLookUp.cu:108-125,
// kmeans.cu:131-135).
inline uint32_t nearest(const uint8_t* x, const uint8_t* nodeCenters, uint32_t B)
{
    uint32_t best = 0;
    uint32_t bestD = dist128(x, nodeCenters);
    for (uint32_t b = 1; b < B; b++) {
        const uint32_t d = dist128(x, nodeCenters + size_t(b) * kDims);
        if (d < bestD) {
            bestD = d;
            best = b;
        }
    }
    return best;
}

__attribute__((target_clones("arch=skylake-avx512", "avx2", "default")))
void lookupRange(const uint8_t* centers, uint32_t B, uint32_t L, const uint8_t* desc, uint64_t beg,
                 uint64_t end, uint32_t* out)
{
    for (uint64_t i = beg; i < end; i++) {
        const uint8_t* x = desc + i * kDims;
        uint64_t idx = 0;
        uint64_t lb = 0; // levelBeg(level)
        for (uint32_t level = 0; level < L; level++) {
            const uint8_t* node = centers + (lb + idx) * B * kDims;
            uint32_t best = 0;
            uint32_t bestD = 0;
            for (uint32_t b = 0; b < B; b++) {
                uint32_t acc = 0;
                const uint8_t* c = node + size_t(b) * kDims;
                for (uint32_t k = 0; k < kDims; k++) {
                    const int d = int(x[k]) - int(c[k]);
                    acc += uint32_t(d * d);
                }
                if (b == 0 || acc < bestD) {
                    bestD = acc;
                    best = b;
                }
            }
            idx = idx * B + best; // FullTree::gotoChild (FullTree.h:59-61)
            lb = lb * B + 1;
        }
        out[i] = static_cast<uint32_t>(idx);
    }
}

// ------------------------------------------------------------------ k-means pieces

// Update of one center set (kmeans.cu:356-372), IEEE division (see header).
void updateCenters(const uint32_t* counts, const uint64_t* sums, uint32_t B, uint8_t* centers)
{
    for (uint32_t b = 0; b < B; b++) {
        if (counts[b] == 0) continue;
        for (uint32_t k = 0; k < kDims; k++) {
            const float q = float(sums[size_t(b) * kDims + k]) / float(counts[b]);
            centers[size_t(b) * kDims + k] = static_cast<uint8_t>(std::round(q));
        }
    }
}

void assignNode(const uint8_t* desc, const uint32_t* members, uint32_t n, const uint8_t* centers, uint32_t B,
                uint8_t* assign, uint32_t* counts, uint64_t* sums, uint32_t* nbChanged)
{
    for (uint32_t i = 0; i < n; i++) {
        const uint8_t* x = desc + size_t(members[i]) * kDims;
        const uint32_t b = nearest(x, centers, B);
        if (assign[i] != b) (*nbChanged)++;
        assign[i] = static_cast<uint8_t>(b);
        counts[b]++;
        for (uint32_t k = 0; k < kDims; k++) sums[size_t(b) * kDims + k] += x[k];
    }
}

// randPick (kmeans.cpp:141-168): min(n, nbToPick) distinct random members, sorted, padded with
// the last pick.  `rng` is the caller's state (the reference keeps one thread_local engine).
uint32_t randPick(std::mt19937_64& rng, uint32_t* dst, uint32_t randSpace, uint32_t nbToPick)
{
    const uint32_t nbPick = std::min(randSpace, nbToPick);
    if (nbPick * 16 < randSpace) {
        std::unordered_set<uint32_t> results;
        while (results.size() != nbPick) results.insert(static_cast<uint32_t>(rng() % randSpace));
        std::copy_n(results.begin(), nbPick, dst);
        std::sort(dst, dst + nbPick);
    } else {
        std::vector<uint32_t> space(randSpace);
        std::iota(space.begin(), space.end(), 0u);
        std::shuffle(space.begin(), space.end(), rng);
        std::copy_n(space.begin(), nbPick, dst);
        std::sort(dst, dst + nbPick);
    }
    if (nbPick < nbToPick) std::fill(dst + nbPick, dst + nbToPick, nbPick != 0 ? dst[nbPick - 1u] : 0u);
    return nbPick;
}

uint64_t splitmix64(uint64_t& s)
{
    // SplitMix64 (Steele, Lea, Flood 2014; constants as published by Vigna).
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

} // namespace

extern "C" {

uint64_t orc_level_beg(uint32_t B, uint32_t level) { return levelBeg(B, level); }

void orc_lookup(const uint8_t* centers, uint32_t B, uint32_t L, const uint8_t* desc, uint64_t n, uint32_t* out,
                uint32_t nThreads)
{
    if (nThreads <= 1 || n < 4096) {
        lookupRange(centers, B, L, desc, 0, n, out);
        return;
    }
    std::vector<std::thread> pool;
    const uint64_t chunk = (n + nThreads - 1) / nThreads;
    for (uint32_t t = 0; t < nThreads; t++) {
        const uint64_t beg = std::min<uint64_t>(n, chunk * t);
        const uint64_t end = std::min<uint64_t>(n, beg + chunk);
        pool.emplace_back([=] { lookupRange(centers, B, L, desc, beg, end, out); });
    }
    for (auto& th : pool) th.join();
}

void orc_kmeans_assign(const uint8_t* desc, const uint32_t* members, uint32_t n, const uint8_t* centers, uint32_t B,
                       uint8_t* assign, uint32_t* counts, uint64_t* sums, uint32_t* nbChanged)
{
    assignNode(desc, members, n, centers, B, assign, counts, sums, nbChanged);
}

void orc_kmeans_update(const uint32_t* counts, const uint64_t* sums, uint32_t B, uint8_t* centers)
{
    updateCenters(counts, sums, B, centers);
}

uint32_t orc_kmeanspp_init(const uint8_t* desc, const uint32_t* members, uint32_t n, uint32_t B, uint64_t seed,
                           uint32_t level, uint64_t nodeInLevel, uint32_t* pickedDesc)
{
    // Seeded k-means++ over at most 256 sampled members (the scheme kmeans.cpp:182-183 sketches).
    uint64_t s = seed ^ (uint64_t(level) * 0x9E3779B97F4A7C15ull) ^ (nodeInLevel * 0xD1B54A32D192ED03ull);
    if (n == 0) {
        for (uint32_t b = 0; b < B; b++) pickedDesc[b] = kInvalid;
        return 0;
    }
    const uint32_t S = std::min<uint32_t>(n, 256);
    std::vector<uint32_t> pos;
    pos.reserve(S);
    if (n <= 256) {
        for (uint32_t i = 0; i < n; i++) pos.push_back(i);
    } else {
        // Floyd's sampling without replacement.
        for (uint32_t j = n - S; j < n; j++) {
            const uint32_t t = static_cast<uint32_t>(splitmix64(s) % (uint64_t(j) + 1));
            if (std::find(pos.begin(), pos.end(), t) == pos.end()) {
                pos.push_back(t);
            } else {
                pos.push_back(j);
            }
        }
        std::sort(pos.begin(), pos.end());
    }
    std::vector<uint32_t> cand(S);
    for (uint32_t i = 0; i < S; i++) cand[i] = members[pos[i]];
    std::vector<uint64_t> d2(S);
    std::vector<uint32_t> chosen;
    chosen.push_back(static_cast<uint32_t>(splitmix64(s) % S));
    for (uint32_t i = 0; i < S; i++)
        d2[i] = dist128(desc + size_t(cand[i]) * kDims, desc + size_t(cand[chosen[0]]) * kDims);
    while (chosen.size() < B) {
        uint64_t total = 0;
        for (uint32_t i = 0; i < S; i++) total += d2[i];
        if (total == 0) break;
        const uint64_t t = splitmix64(s) % total;
        uint64_t prefix = 0;
        uint32_t pick = S - 1;
        for (uint32_t i = 0; i < S; i++) {
            prefix += d2[i];
            if (prefix > t) {
                pick = i;
                break;
            }
        }
        chosen.push_back(pick);
        for (uint32_t i = 0; i < S; i++) {
            const uint64_t d = dist128(desc + size_t(cand[i]) * kDims, desc + size_t(cand[pick]) * kDims);
            d2[i] = std::min(d2[i], d);
        }
    }
    const uint32_t nValid = static_cast<uint32_t>(chosen.size());
    for (uint32_t b = 0; b < B; b++) pickedDesc[b] = cand[chosen[std::min(b, nValid - 1)]];
    return nValid;
}

int orc_build_vocabulary(const uint8_t* desc, uint32_t nbDesc, uint32_t nbDoc, uint32_t B, uint32_t L,
                         uint32_t maxIter, uint32_t initMode, uint64_t seed, const uint32_t* injected,
                         uint8_t* centers, uint32_t* masks, float* weights, uint32_t* occ, uint32_t* itersOut)
{
    if (nbDesc < B || nbDoc == 0 || B < 2 || B > 16) return -1; // Vocabulary.cpp:39-44
    const uint64_t nbNodes = levelBeg(B, L);
    std::fill(masks, masks + nbNodes, 0u);
    std::fill(occ, occ + nbNodes * B, 0u);
    std::mt19937_64 rng{}; // kmeans.cpp:145, a fresh thread's engine
    // Groups of the current level, in breadth-first order (Vocabulary.cpp:50-52).
    std::vector<std::vector<uint32_t>> groups{std::vector<uint32_t>(nbDesc)};
    std::iota(groups[0].begin(), groups[0].end(), 0u);
    for (uint32_t level = 0; level < L; level++) {
        const uint64_t lb = levelBeg(B, level);
        const uint64_t nbGroups = groups.size();
        std::vector<std::vector<uint32_t>> next(nbGroups * B);
        for (uint64_t g = 0; g < nbGroups; g++) {
            const auto& members = groups[g];
            const uint32_t n = static_cast<uint32_t>(members.size());
            uint8_t* c = centers + (lb + g) * B * kDims;
            // ---- initial centers
            std::vector<uint32_t> picks(B, kInvalid);
            uint32_t nValid = 0;
            if (initMode == ORC_INIT_REFERENCE) {
                // makeRandCenters (kmeans.cpp:170-196) + launchKMeansInitCenters (reformatDesc.cu:88-96)
                std::vector<uint32_t> tmp(B);
                nValid = randPick(rng, tmp.data(), n, B);
                if (n != 0) {
                    for (uint32_t b = 0; b < B; b++) picks[b] = members[tmp[b]];
                } else {
                    // An empty group reads grpIndices[0] at its padded offset (kmeans.cpp:179-186):
                    // the first member of the next non-empty group of this level, if any.
                    uint32_t v = kInvalid;
                    for (uint64_t h = g + 1; h < nbGroups; h++) {
                        if (!groups[h].empty()) {
                            v = groups[h][0];
                            break;
                        }
                    }
                    for (uint32_t b = 0; b < B; b++) picks[b] = v;
                }
            } else if (initMode == ORC_INIT_KMEANSPP) {
                nValid = orc_kmeanspp_init(desc, members.data(), n, B, seed, level, g, picks.data());
            } else {
                for (uint32_t b = 0; b < B; b++) {
                    picks[b] = injected[(lb + g) * B + b];
                    if (picks[b] != kInvalid && b == nValid) nValid++;
                }
            }
            for (uint32_t b = 0; b < B; b++) {
                if (picks[b] == kInvalid) {
                    std::memset(c + size_t(b) * kDims, 0xFF, kDims);
                } else {
                    std::memcpy(c + size_t(b) * kDims, desc + size_t(picks[b]) * kDims, kDims);
                }
            }
            masks[lb + g] = nValid >= 32 ? 0xFFFFFFFFu : ((1u << nValid) - 1u);
            // ---- Lloyd iterations (kmeans.cpp:118-133 with kmeans.cu:238-240,341-343):
            // a node whose last iteration changed nothing is frozen; the convergence-check
            // interval only decides when the host stops and does not change any node's result.
            std::vector<uint8_t> assign(n, 0); // fresh (zeroed) assignment memory
            std::vector<uint32_t> counts(B);
            std::vector<uint64_t> sums(size_t(B) * kDims);
            uint32_t last = 0xFFFFFFFFu;
            uint32_t iters = 0;
            for (uint32_t it = 0; it < maxIter; it++) {
                uint32_t changed = 0;
                std::fill(counts.begin(), counts.end(), 0u);
                std::fill(sums.begin(), sums.end(), 0ull);
                if (last != 0) {
                    assignNode(desc, members.data(), n, c, B, assign.data(), counts.data(), sums.data(), &changed);
                    iters = it + 1;
                }
                if (changed == 0) break;
                updateCenters(counts.data(), sums.data(), B, c);
                last = changed;
            }
            if (itersOut) itersOut[lb + g] = iters;
            // ---- stable regroup by assignment (Vocabulary.cpp:83-98)
            for (uint32_t i = 0; i < n; i++) next[g * B + assign[i]].push_back(members[i]);
            for (uint32_t b = 0; b < B; b++) occ[(lb + g) * B + b] = static_cast<uint32_t>(next[g * B + b].size());
        }
        groups.swap(next);
    }
    // idf-like weights (Vocabulary.cpp:103-108)
    for (uint64_t i = 0; i < nbNodes * B; i++) {
        weights[i] = occ[i] == 0 ? std::numeric_limits<float>::min()
                                 : std::max(std::numeric_limits<float>::min(),
                                            std::log(float(nbDoc) / float(occ[i])));
    }
    return 0;
}

} // extern "C"

// ------------------------------------------------------------------ float-center mode
namespace {

// orc_dist64's evaluation order: 32 lane partials of four fused multiply-adds, then a butterfly
// of pairwise sums (each level adds the partner that differs in one index bit; the sums are
// symmetric, so lane l < off keeps p_l + p_(l+off)).  Operands come "lane-major transposed":
// v[32 k + l] holds element 4 l + k, so every step is a contiguous vector operation.
static inline __attribute__((always_inline)) double dist64T(const double* __restrict__ xT,
                                                           const double* __restrict__ cT)
{
    double p[32];
    for (uint32_t l = 0; l < 32; l++) p[l] = 0.0;
    for (uint32_t k = 0; k < 4; k++) {
        for (uint32_t l = 0; l < 32; l++) {
            const double e = xT[32 * k + l] - cT[32 * k + l];
            p[l] = std::fma(e, e, p[l]);
        }
    }
    for (uint32_t off = 16; off > 0; off >>= 1)
        for (uint32_t l = 0; l < off; l++) p[l] = p[l] + p[l + off];
    return p[0];
}

template <typename T>
static inline __attribute__((always_inline)) void transposeToDouble(const T* v, double* out)
{
    for (uint32_t l = 0; l < 32; l++)
        for (uint32_t k = 0; k < 4; k++) out[32 * k + l] = double(v[4 * l + k]);
}

double dist64(const uint8_t* x, const float* c)
{
    double xT[kDims], cT[kDims];
    transposeToDouble(x, xT);
    transposeToDouble(c, cT);
    return dist64T(xT, cT);
}

// argmin over the B transposed centers cT[B][128], lowest index on ties.
static inline __attribute__((always_inline)) uint32_t nearestT(const uint8_t* x, const double* cT, uint32_t B,
                                                               double* dOut)
{
    double xT[kDims];
    transposeToDouble(x, xT);
    uint32_t best = 0;
    double bestD = dist64T(xT, cT);
    for (uint32_t b = 1; b < B; b++) {
        const double d = dist64T(xT, cT + size_t(b) * kDims);
        if (d < bestD) {
            bestD = d;
            best = b;
        }
    }
    if (dOut) *dOut = bestD;
    return best;
}

void transposeCenters(const float* c, uint32_t B, std::vector<double>& cT)
{
    cT.resize(size_t(B) * kDims);
    for (uint32_t b = 0; b < B; b++) transposeToDouble(c + size_t(b) * kDims, cT.data() + size_t(b) * kDims);
}

// Nearest fp32 center (transposed cT[B][128]) of members[beg, end): assignment and distance.
__attribute__((target_clones("avx512f", "fma", "default")))
void assignRangeF(const uint8_t* desc, const uint32_t* members, uint32_t beg, uint32_t end, const double* cT,
                  uint32_t B, uint8_t* next, double* dist)
{
    for (uint32_t i = beg; i < end; i++)
        next[i] = static_cast<uint8_t>(nearestT(desc + size_t(members[i]) * kDims, cT, B, &dist[i]));
}

// Descent of desc[beg, end) through fp32 centers [levelBeg(L)][B][128].
__attribute__((target_clones("avx512f", "fma", "default")))
void lookupRangeF(const float* centers, uint32_t B, uint32_t L, const uint8_t* desc, uint64_t beg, uint64_t end,
                  uint32_t* out)
{
    std::vector<double> cT(size_t(B) * kDims);
    for (uint64_t i = beg; i < end; i++) {
        const uint8_t* x = desc + i * kDims;
        uint64_t idx = 0, lb = 0;
        for (uint32_t level = 0; level < L; level++) {
            const float* node = centers + (lb + idx) * B * kDims;
            for (uint32_t b = 0; b < B; b++) transposeToDouble(node + size_t(b) * kDims, cT.data() + size_t(b) * kDims);
            idx = idx * B + nearestT(x, cT.data(), B, nullptr);
            lb = lb * B + 1;
        }
        out[i] = static_cast<uint32_t>(idx);
    }
}

template <typename F>
void parallelFor(uint64_t n, uint32_t nThreads, F&& f)
{
    if (nThreads <= 1 || n < 2) {
        for (uint64_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> pool;
    const uint32_t m = static_cast<uint32_t>(std::min<uint64_t>(nThreads, n));
    for (uint32_t t = 0; t < m; t++) {
        pool.emplace_back([&] {
            for (;;) {
                const uint64_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i);
            }
        });
    }
    for (auto& th : pool) th.join();
}

// Initial descriptor picks of every node of one level (the uint8 build's rules), in node order
// because the reference init draws from one engine across the level.
void levelInitPicks(uint32_t initMode, std::mt19937_64& rng, const uint8_t* desc,
                    const std::vector<std::vector<uint32_t>>& groups, uint32_t B, uint64_t seed, uint32_t level,
                    uint64_t lb, const uint32_t* injected, std::vector<uint32_t>& picks, std::vector<uint32_t>& nValid)
{
    const uint64_t nbGroups = groups.size();
    picks.assign(nbGroups * B, kInvalid);
    nValid.assign(nbGroups, 0u);
    for (uint64_t g = 0; g < nbGroups; g++) {
        const auto& members = groups[g];
        const uint32_t n = static_cast<uint32_t>(members.size());
        uint32_t* pk = picks.data() + g * B;
        if (initMode == ORC_INIT_REFERENCE) {
            std::vector<uint32_t> tmp(B);
            nValid[g] = randPick(rng, tmp.data(), n, B);
            if (n != 0) {
                for (uint32_t b = 0; b < B; b++) pk[b] = members[tmp[b]];
            } else {
                uint32_t v = kInvalid;
                for (uint64_t h = g + 1; h < nbGroups; h++) {
                    if (!groups[h].empty()) {
                        v = groups[h][0];
                        break;
                    }
                }
                for (uint32_t b = 0; b < B; b++) pk[b] = v;
            }
        } else if (initMode == ORC_INIT_KMEANSPP) {
            nValid[g] = orc_kmeanspp_init(desc, members.data(), n, B, seed, level, g, pk);
        } else {
            for (uint32_t b = 0; b < B; b++) {
                pk[b] = injected[(lb + g) * B + b];
                if (pk[b] != kInvalid && b == nValid[g]) nValid[g]++;
            }
        }
    }
}

struct NodeRunF {
    uint32_t iters = 0;
    double inertiaFirst = 0;
    double inertiaLast = 0;
};

// Lloyd iterations of one node with fp32 centers (kmeans.cu:125-199 and 356-372 generalised,
// freezing as kmeans.cu:238-240 / 341-343).  innerThreads > 1 splits the members' distances
// over threads; every reduction is in member order, so the result does not depend on it.
NodeRunF runNodeF(const uint8_t* desc, const std::vector<uint32_t>& members, uint32_t B, uint32_t maxIter, float* c,
                  std::vector<uint8_t>& assign, uint32_t innerThreads)
{
    NodeRunF r;
    const uint32_t n = static_cast<uint32_t>(members.size());
    assign.assign(n, 0);
    std::vector<uint8_t> next(n);
    std::vector<double> dist(n);
    std::vector<uint32_t> counts(B);
    std::vector<uint64_t> sums(size_t(B) * kDims);
    uint32_t last = 0xFFFFFFFFu;
    constexpr uint32_t kChunk = 4096;
    std::vector<double> cT;
    for (uint32_t it = 0; it < maxIter; it++) {
        uint32_t changed = 0;
        if (last != 0) {
            transposeCenters(c, B, cT);
            parallelFor((n + kChunk - 1) / kChunk, innerThreads, [&](uint64_t ch) {
                const uint32_t beg = static_cast<uint32_t>(ch * kChunk);
                assignRangeF(desc, members.data(), beg, std::min(n, beg + kChunk), cT.data(), B, next.data(),
                             dist.data());
            });
            std::fill(counts.begin(), counts.end(), 0u);
            std::fill(sums.begin(), sums.end(), 0ull);
            double inertia = 0.0;
            for (uint32_t i = 0; i < n; i++) {
                if (next[i] != assign[i]) changed++;
                assign[i] = next[i];
                counts[next[i]]++;
                const uint8_t* x = desc + size_t(members[i]) * kDims;
                uint64_t* s = sums.data() + size_t(next[i]) * kDims;
                for (uint32_t k = 0; k < kDims; k++) s[k] += x[k];
                inertia += dist[i];
            }
            if (it == 0) r.inertiaFirst = inertia;
            r.inertiaLast = inertia;
            r.iters = it + 1;
        }
        if (changed == 0) break;
        for (uint32_t b = 0; b < B; b++) {
            if (counts[b] == 0) continue;
            for (uint32_t k = 0; k < kDims; k++)
                c[size_t(b) * kDims + k] = float(double(sums[size_t(b) * kDims + k]) / double(counts[b]));
        }
        last = changed;
    }
    return r;
}

} // namespace

extern "C" {

double orc_dist64(const uint8_t* x, const float* c) { return dist64(x, c); }

void orc_lookup_f32(const float* centers, uint32_t B, uint32_t L, const uint8_t* desc, uint64_t n, uint32_t* out,
                    uint32_t nThreads)
{
    constexpr uint64_t kChunk = 2048;
    parallelFor((n + kChunk - 1) / kChunk, nThreads, [&](uint64_t ch) {
        const uint64_t beg = ch * kChunk;
        lookupRangeF(centers, B, L, desc, beg, std::min(n, beg + kChunk), out);
    });
}

int orc_build_vocabulary_f32(const uint8_t* desc, uint32_t nbDesc, uint32_t nbDoc, uint32_t B, uint32_t L,
                             uint32_t maxIter, uint32_t initMode, uint64_t seed, const uint32_t* injected,
                             float* centers, uint32_t* masks, float* weights, uint32_t* occ, uint32_t* itersOut,
                             double* inertiaFirst, double* inertiaLast, uint32_t nThreads)
{
    if (nbDesc < B || nbDoc == 0 || B < 2 || B > 16) return -1;
    const uint64_t nbNodes = levelBeg(B, L);
    std::fill(masks, masks + nbNodes, 0u);
    std::fill(occ, occ + nbNodes * B, 0u);
    std::mt19937_64 rng{};
    std::vector<std::vector<uint32_t>> groups{std::vector<uint32_t>(nbDesc)};
    std::iota(groups[0].begin(), groups[0].end(), 0u);
    std::vector<uint32_t> picks, nValid;
    for (uint32_t level = 0; level < L; level++) {
        const uint64_t lb = levelBeg(B, level);
        const uint64_t nbGroups = groups.size();
        levelInitPicks(initMode, rng, desc, groups, B, seed, level, lb, injected, picks, nValid);
        for (uint64_t g = 0; g < nbGroups; g++) {
            float* c = centers + (lb + g) * B * kDims;
            for (uint32_t b = 0; b < B; b++) {
                const uint32_t pk = picks[g * B + b];
                for (uint32_t k = 0; k < kDims; k++)
                    c[size_t(b) * kDims + k] = pk == kInvalid ? 255.0f : float(desc[size_t(pk) * kDims + k]);
            }
            masks[lb + g] = nValid[g] >= 32 ? 0xFFFFFFFFu : ((1u << nValid[g]) - 1u);
        }
        std::vector<NodeRunF> runs(nbGroups);
        std::vector<std::vector<uint8_t>> assigns(nbGroups);
        const bool manyNodes = nbGroups >= 4ull * std::max(1u, nThreads);
        parallelFor(nbGroups, manyNodes ? nThreads : 1u, [&](uint64_t g) {
            runs[g] = runNodeF(desc, groups[g], B, maxIter, centers + (lb + g) * B * kDims, assigns[g],
                               manyNodes ? 1u : nThreads);
        });
        double first = 0.0, lastSum = 0.0;
        std::vector<std::vector<uint32_t>> next(nbGroups * B);
        for (uint64_t g = 0; g < nbGroups; g++) {
            first += runs[g].inertiaFirst;
            lastSum += runs[g].inertiaLast;
            if (itersOut) itersOut[lb + g] = runs[g].iters;
            const auto& members = groups[g];
            for (size_t i = 0; i < members.size(); i++) next[g * B + assigns[g][i]].push_back(members[i]);
            for (uint32_t b = 0; b < B; b++) occ[(lb + g) * B + b] = static_cast<uint32_t>(next[g * B + b].size());
        }
        if (inertiaFirst) inertiaFirst[level] = first;
        if (inertiaLast) inertiaLast[level] = lastSum;
        groups.swap(next);
    }
    for (uint64_t i = 0; i < nbNodes * B; i++) {
        weights[i] = occ[i] == 0 ? std::numeric_limits<float>::min()
                                 : std::max(std::numeric_limits<float>::min(),
                                            std::log(float(nbDoc) / float(occ[i])));
    }
    return 0;
}

} // extern "C"

// ------------------------------------------------------------------ DataBase restatement
namespace {
struct OrcDb {
    uint32_t B;
    uint32_t L;
    std::vector<float> weights;                   // [levelBeg(L)][B]
    std::vector<std::vector<uint32_t>> postings;  // per leaf word, sorted with duplicates
    std::map<uint32_t, float> rcpF;               // DataBase.h:62
    std::map<uint32_t, double> rcpD;              // FP64 restatement
    std::vector<uint64_t> extWordPost;            // skip-rule counts set from outside (empty: own)

    const float* levelWeights(uint32_t level) const { return &weights[levelBeg(B, level) * B]; }

    // L1 norm of the weight vector over all levels (DataBase.cpp:54-67, 77-94), double sum in the
    // reference order: levels leaf->root, descriptors in ascending leaf order.
    double l1norm(const uint32_t* leaves, uint32_t n) const
    {
        std::vector<uint64_t> idx(leaves, leaves + n);
        std::sort(idx.begin(), idx.end());
        double norm = 0;
        for (uint32_t it = 0; it < L; it++) {
            const uint32_t level = L - 1 - it;
            const float* lw = levelWeights(level);
            for (uint32_t i = 0; i < n; i++) {
                norm += lw[idx[i]];
                idx[i] /= B;
            }
        }
        return norm;
    }
};
} // namespace

extern "C" {

void* orc_db_create(uint32_t B, uint32_t L, const float* weights)
{
    auto* db = new OrcDb{};
    db->B = B;
    db->L = L;
    db->weights.assign(weights, weights + levelBeg(B, L) * B);
    db->postings.resize(ipow(B, L));
    return db;
}

void orc_db_destroy(void* db) { delete static_cast<OrcDb*>(db); }

int orc_db_add(void* p, uint32_t idxDoc, const uint32_t* leaves, uint32_t n)
{
    auto* db = static_cast<OrcDb*>(p);
    if (db->rcpF.count(idxDoc)) return -1; // DataBase.cpp:41-43
    for (uint32_t i = 0; i < n; i++) {
        auto& ivf = db->postings.at(leaves[i]);
        ivf.insert(std::upper_bound(ivf.begin(), ivf.end(), idxDoc), idxDoc); // DataBase.cpp:44-53
    }
    const double norm = db->l1norm(leaves, n);
    db->rcpF[idxDoc] = float(1 / norm);
    db->rcpD[idxDoc] = 1 / norm;
    return 0;
}

float orc_db_doc_rcp(const void* p, uint32_t idxDoc)
{
    const auto* db = static_cast<const OrcDb*>(p);
    const auto it = db->rcpF.find(idxDoc);
    return it == db->rcpF.end() ? -1.f : it->second;
}

void orc_db_word_postings(const void* p, uint64_t* out)
{
    const auto* db = static_cast<const OrcDb*>(p);
    for (uint32_t level = 0; level < db->L; level++) {
        const uint64_t span = ipow(db->B, db->L - 1 - level);
        const uint64_t words = ipow(db->B, level + 1);
        for (uint64_t w = 0; w < words; w++) {
            uint64_t total = 0;
            for (uint64_t f = w * span; f < (w + 1) * span; f++) total += db->postings[f].size();
            out[levelBeg(db->B, level) * db->B + w] = total;
        }
    }
}

void orc_db_set_word_postings(void* p, const uint64_t* counts)
{
    auto* db = static_cast<OrcDb*>(p);
    if (counts == nullptr) {
        db->extWordPost.clear();
        return;
    }
    db->extWordPost.assign(counts, counts + levelBeg(db->B, db->L) * db->B);
}

uint32_t orc_db_postings(const void* p, uint32_t leaf, uint32_t* out, uint32_t capacity)
{
    const auto& ivf = static_cast<const OrcDb*>(p)->postings.at(leaf);
    const uint32_t n = std::min<uint32_t>(capacity, static_cast<uint32_t>(ivf.size()));
    std::copy_n(ivf.begin(), n, out);
    return static_cast<uint32_t>(ivf.size());
}

uint32_t orc_db_query(const void* p, const uint32_t* leaves, uint32_t n, uint32_t maxNbResults, int mode,
                      uint32_t* docs, double* scores, uint32_t capacity)
{
    const auto* db = static_cast<const OrcDb*>(p);
    const uint32_t B = db->B;
    const uint32_t L = db->L;
    const double qNorm = db->l1norm(leaves, n);
    const float qRcpF = float(1 / qNorm);
    const double qRcpD = 1 / qNorm;
    std::vector<uint32_t> sorted(leaves, leaves + n);
    std::sort(sorted.begin(), sorted.end());
    std::map<uint32_t, double> acc;
    for (uint32_t it = 0; it < L; it++) { // DataBase.cpp:103-169
        const uint32_t level = L - 1 - it;
        const float* lw = db->levelWeights(level);
        const uint64_t span = ipow(B, it); // leaf inverted files under one word of this level
        for (uint32_t i = 0; i < n;) {
            const uint64_t node = sorted[i] / span;
            uint32_t run = 1;
            while (i + run < n && sorted[i + run] / span == node) run++;
            const float w = lw[node];
            const uint64_t leafBeg = node * span;
            uint64_t total = 0;
            if (db->extWordPost.empty()) {
                for (uint64_t f = leafBeg; f < leafBeg + span; f++) total += db->postings[f].size();
            } else {
                total = db->extWordPost[levelBeg(B, level) * B + node];
            }
            if (level >= L - 1 || total < 16u + uint64_t(maxNbResults) * 4u) { // DataBase.cpp:125
                std::map<uint32_t, uint32_t> cnt;
                for (uint64_t f = leafBeg; f < leafBeg + span; f++)
                    for (const uint32_t d : db->postings[f]) cnt[d]++;
                for (const auto& [doc, c] : cnt) {
                    if (mode == 0) {
                        const float q = float(run) * w * qRcpF;
                        const float d = float(c) * w * db->rcpF.at(doc);
                        acc[doc] += std::abs(q - d) - (q + d);
                    } else {
                        const double q = double(run) * double(w) * qRcpD;
                        const double d = double(c) * double(w) * db->rcpD.at(doc);
                        acc[doc] += std::abs(q - d) - (q + d);
                    }
                }
            }
            i += run;
        }
    }
    std::vector<std::pair<double, uint32_t>> order;
    order.reserve(acc.size());
    for (const auto& [doc, a] : acc) {
        const double s = mode == 0 ? double(float(a + 2.f)) : a + 2.0; // DataBase.cpp:170-174
        order.emplace_back(s, doc);
    }
    std::sort(order.begin(), order.end());
    const uint32_t m = std::min<uint32_t>(capacity, static_cast<uint32_t>(order.size()));
    for (uint32_t i = 0; i < m; i++) {
        docs[i] = order[i].second;
        scores[i] = order[i].first;
    }
    return static_cast<uint32_t>(order.size());
}

} // extern "C"
