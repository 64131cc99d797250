// Retrieval serving loop: continuous batching of query images over a device-resident DataBase.
//
// A request is one query image's descriptors (host memory).  Requests are answered with the
// image's top-k database documents, computed as the reference's application does it: the
// descriptors are looked up to leaf words (IVocabulary::lookUp, Vocabulary.cpp:162-173) and the
// words scored against the inverted file (DataBase::query, DataBase.cpp:71-190).
//
// Batching: a dispatcher thread forms a batch from the pending requests, in arrival order, as
// soon as a batch slot is free, up to the slot's request and descriptor limits and only while
// the batch's device memory estimate fits the memory budget left by the batches in flight
// (admission by free HBM).  A request's descriptors are copied once, at submit, into a pinned
// buffer from a pool; the batch copies each of its requests to the device straight from there
// (one asynchronous copy per request), looks them up and scores all its
// requests in one scoring launch, on its own stream, so up to max_inflight batches overlap on
// the GPU; requests that arrive meanwhile join the next batch.  A completion thread waits for
// each batch in order, hands the results to the requests and frees the slot.
//
// Results do not depend on how requests were batched: the lookup is exact and every query is
// scored independently with an order-independent sum.
#include "capi_internal.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace rbw {
namespace {

using Clock = std::chrono::steady_clock;

// Pinned host buffers in power-of-two size classes (64 KiB and up), reused across requests, so
// a request's descriptors are copied once on the host and DMA-copied to the device from there.
class PinnedPool
{
public:
    ~PinnedPool()
    {
        for (auto& cls : mFree)
            for (void* p : cls) cudaFreeHost(p);
    }
    // Returns a buffer of at least `bytes` and its size class.
    std::pair<uint8_t*, uint32_t> take(size_t bytes)
    {
        uint32_t c = 16;
        while ((size_t(1) << c) < bytes) c++;
        {
            std::lock_guard<std::mutex> lk(mMu);
            if (c < mFree.size() && !mFree[c].empty()) {
                void* p = mFree[c].back();
                mFree[c].pop_back();
                return {static_cast<uint8_t*>(p), c};
            }
        }
        void* p = nullptr;
        RBW_CUDA(cudaMallocHost(&p, size_t(1) << c));
        return {static_cast<uint8_t*>(p), c};
    }
    // Fills each size class from 2^lo to 2^hi bytes with `count` buffers ahead of time, so the
    // first requests do not wait for page-locked allocations.
    void reserve(uint32_t lo, uint32_t hi, uint32_t count)
    {
        for (uint32_t c = lo; c <= hi; c++)
            for (uint32_t k = 0; k < count; k++) {
                void* p = nullptr;
                RBW_CUDA(cudaMallocHost(&p, size_t(1) << c));
                give(static_cast<uint8_t*>(p), c);
            }
    }
    void give(uint8_t* p, uint32_t c)
    {
        if (p == nullptr) return;
        std::lock_guard<std::mutex> lk(mMu);
        if (mFree.size() <= c) mFree.resize(c + 1);
        mFree[c].push_back(p);
    }

private:
    std::mutex mMu;
    std::vector<std::vector<void*>> mFree;
};

struct Request {
    uint64_t id = 0;
    uint8_t* desc = nullptr;     // pinned, n x 128 (from the server's pool)
    uint32_t descClass = 0;
    uint32_t n = 0;
    Clock::time_point submitted, dispatched, launched, finished;
    bool done = false;
    int status = 0;
    std::string error;
    std::vector<uint32_t> docs;
    std::vector<float> scores;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    uint64_t* hOff = nullptr;     // pinned [maxQueries + 1]
    uint32_t* hDocs = nullptr;    // pinned [maxQueries][k]
    float* hScores = nullptr;     // pinned [maxQueries][k]
    uint32_t* hCount = nullptr;   // pinned [maxQueries]
    std::vector<std::shared_ptr<Request>> reqs;
    size_t reserved = 0;
    bool busy = false;
    int status = 0;
    std::string error;
};

class Server
{
public:
    Server(const rbw_vocabulary* voc, rbw_database* db, const rbw_server_options& o) : mVoc{voc}, mDb{db}, mOpt{o}
    {
        if (mOpt.max_batch_queries == 0 || mOpt.max_batch_descriptors == 0 || mOpt.max_inflight_batches == 0)
            throw Error(kInvalidArg, "server limits must be positive");
        if (mOpt.max_results == 0) throw Error(kInvalidArg, "max_results must be positive");
        RBW_CUDA(cudaGetDevice(&mDevice));
        const Vocabulary& v = vocabularyOf(voc);
        mLevels = v.levels();
        if (mOpt.hbm_budget_bytes == 0) {
            size_t freeB = 0, totalB = 0;
            RBW_CUDA(cudaMemGetInfo(&freeB, &totalB));
            mOpt.hbm_budget_bytes = freeB / 2;
        }
        uint32_t nDocs = 0;
        if (rbw_db_info(db, &nDocs, nullptr) != RBW_OK) throw Error(kInvalidArg, rbw_last_error());
        mSlots.resize(mOpt.max_inflight_batches);
        const size_t q = mOpt.max_batch_queries, k = mOpt.max_results;
        for (Slot& s : mSlots) {
            RBW_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
            RBW_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
            RBW_CUDA(cudaMallocHost(&s.hOff, (q + 1) * 8));
            RBW_CUDA(cudaMallocHost(&s.hDocs, q * k * 4));
            RBW_CUDA(cudaMallocHost(&s.hScores, q * k * 4));
            RBW_CUDA(cudaMallocHost(&s.hCount, q * 4));
        }
        {
            // Requests of up to 8,192 descriptors find a pinned buffer ready, 32 per size class
            // (waiting and in-flight requests together): a page-locked allocation during serving
            // is a driver call that can hold up the other threads' CUDA calls for milliseconds.
            uint32_t hi = 16;
            while (hi < 20 && (size_t(1) << hi) < mOpt.max_batch_descriptors * 128) hi++;
            mPinned.reserve(16, hi, 32);
        }
        {
            // Grow the device pool once, to what every slot needs for a batch of up to 65,536
            // descriptors: the pool keeps freed memory, so batches of that size never wait for the
            // pool to grow (a growth is a driver call that holds up the dispatcher).
            const uint64_t warmDesc = std::min<uint64_t>(mOpt.max_batch_descriptors, 65536);
            const uint64_t warmQueries = std::min<uint64_t>(mOpt.max_batch_queries, 64);
            const size_t bytes = std::min<size_t>(2 * estimate(warmDesc, warmQueries) * mSlots.size(),
                                                  mOpt.hbm_budget_bytes);
            void* p = nullptr;
            cudaStream_t s0 = mSlots[0].stream;
            if (cudaMallocFromPoolAsync(&p, bytes, libraryPool(), s0) == cudaSuccess) {
                RBW_CUDA(cudaFreeAsync(p, s0));
            } else {
                cudaGetLastError(); // a smaller pool only means growth later
            }
            RBW_CUDA(cudaStreamSynchronize(s0));
        }
        mDispatcher = std::thread([this] { dispatchLoop(); });
        mCompleter = std::thread([this] { completeLoop(); });
    }

    ~Server()
    {
        {
            std::lock_guard<std::mutex> lk(mMu);
            mStop = true;
        }
        mCv.notify_all();
        mDispatcher.join();
        mCompleter.join();
        for (Slot& s : mSlots) {
            cudaStreamSynchronize(s.stream);
            cudaFreeHost(s.hOff);
            cudaFreeHost(s.hDocs);
            cudaFreeHost(s.hScores);
            cudaFreeHost(s.hCount);
            cudaEventDestroy(s.done);
            cudaStreamDestroy(s.stream);
        }
    }

    uint64_t submit(const uint8_t* desc, uint32_t n)
    {
        if (n && desc == nullptr) throw Error(kInvalidArg, "null descriptors");
        if (n > mOpt.max_batch_descriptors) throw Error(kInvalidArg, "request larger than a batch");
        if (estimate(n, 1) > mOpt.hbm_budget_bytes) throw Error(kOutOfMemory, "request larger than the memory budget");
        auto r = std::make_shared<Request>();
        if (n) {
            std::tie(r->desc, r->descClass) = mPinned.take(size_t(n) * 128);
            std::memcpy(r->desc, desc, size_t(n) * 128);
        }
        r->n = n;
        std::lock_guard<std::mutex> lk(mMu);
        if (mStop) throw Error(kInvalidArg, "server stopped");
        r->id = ++mNextId;
        r->submitted = Clock::now();
        mPending.push_back(r);
        mAll.emplace(r->id, r);
        mSubmitted++;
        mCv.notify_all();
        return r->id;
    }

    // Waits for a request (timeout_us < 0: no limit).  Returns false on timeout.
    bool wait(uint64_t id, int64_t timeoutUs, uint32_t* docs, float* scores, uint32_t capacity, uint32_t* nOut,
              double* latencyMs)
    {
        std::unique_lock<std::mutex> lk(mMu);
        auto it = mAll.find(id);
        if (it == mAll.end()) throw Error(kInvalidArg, "unknown request id (already collected?)");
        std::shared_ptr<Request> r = it->second;
        auto ready = [&] { return r->done; };
        if (timeoutUs < 0) {
            mDoneCv.wait(lk, ready);
        } else if (!mDoneCv.wait_for(lk, std::chrono::microseconds(timeoutUs), ready)) {
            return false;
        }
        mAll.erase(it);
        if (r->status != RBW_OK) throw Error(static_cast<Status>(r->status), r->error);
        const uint32_t n = static_cast<uint32_t>(r->docs.size());
        if (nOut) *nOut = n;
        const uint32_t m = std::min(n, capacity);
        if (docs) std::memcpy(docs, r->docs.data(), size_t(m) * 4);
        if (scores) std::memcpy(scores, r->scores.data(), size_t(m) * 4);
        if (latencyMs) *latencyMs = std::chrono::duration<double, std::milli>(r->finished - r->submitted).count();
        return true;
    }

    void stats(rbw_server_stats* st)
    {
        std::lock_guard<std::mutex> lk(mMu);
        std::memset(st, 0, sizeof(*st));
        st->submitted = mSubmitted;
        st->completed = mLatencies.size();
        st->batches = mBatches;
        st->max_inflight_seen = mMaxInflight;
        st->mean_batch_requests = mBatches ? double(mBatchedRequests) / double(mBatches) : 0.0;
        if (!mLatencies.empty()) {
            auto pct = [](std::vector<double> l, double p) {
                const size_t i = std::min(l.size() - 1, static_cast<size_t>(p * double(l.size() - 1) + 0.5));
                std::nth_element(l.begin(), l.begin() + i, l.end());
                return l[i];
            };
            auto maxOf = [](const std::vector<double>& l) { return *std::max_element(l.begin(), l.end()); };
            st->p50_ms = pct(mLatencies, 0.50);
            st->p99_ms = pct(mLatencies, 0.99);
            st->max_ms = maxOf(mLatencies);
            st->queue_p99_ms = pct(mStage[0], 0.99);
            st->launch_p99_ms = pct(mStage[1], 0.99);
            st->device_p99_ms = pct(mStage[2], 0.99);
            st->queue_max_ms = maxOf(mStage[0]);
            st->launch_max_ms = maxOf(mStage[1]);
            st->device_max_ms = maxOf(mStage[2]);
        }
    }

    size_t batchBytes(uint64_t desc, uint64_t queries) const { return estimate(desc, queries); }

    void resetStats()
    {
        std::lock_guard<std::mutex> lk(mMu);
        mLatencies.clear();
        for (auto& v : mStage) v.clear();
        mBatches = mBatchedRequests = 0;
        mMaxInflight = 0;
        mSubmitted = 0;
    }

private:
    // Device bytes a batch of `desc` descriptors in `queries` requests needs: descriptors and
    // leaves, lookup working memory, scoring entries, results and the per-shard candidates of
    // databases scored by several CTAs per query (at most one per 2,560 documents), plus 1 MiB
    // of slack.
    size_t estimate(uint64_t desc, uint64_t queries) const
    {
        uint64_t scratch = 0;
        rbw_voc_lookup_scratch_bytes(mVoc, desc, &scratch);
        uint32_t nDocs = 0;
        rbw_db_info(mDb, &nDocs, nullptr);
        const uint64_t shards = (uint64_t(nDocs) + 2559) / 2560;
        const uint64_t cand = shards > 1 ? queries * shards * mOpt.max_results * 8ull : 0;
        return size_t(desc * (128 + 4 + 16ull * mLevels) + scratch + queries * (mOpt.max_results * 8ull + 32) + cand +
                      (1u << 20));
    }

    // Device memory free right now: the driver's free memory plus what the library's pool holds
    // unused (memory freed by finished batches stays in the pool for the next ones).  The driver
    // is asked at most every kLiveRefresh; in between, the value goes down by what the batches
    // admitted since then reserve.
    static constexpr std::chrono::microseconds kLiveRefresh{500};
    size_t liveFreeBytes()
    {
        const auto now = Clock::now();
        if (now - mLiveAt < kLiveRefresh) return mLiveFree;
        size_t freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return 0;
        cudaMemPool_t pool = libraryPool();
        uint64_t reserved = 0, used = 0;
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
        mLiveFree = freeB + (reserved > used ? size_t(reserved - used) : 0);
        mLiveAt = now;
        return mLiveFree;
    }

    // A batch of `bytes` is admitted while it fits what the batches in flight leave of the budget
    // and the device memory free right now (less kLiveHeadroom).  With nothing in flight the
    // live check is skipped, so memory held by other users cannot stall the queue; the batch
    // then fails with RBW_ERR_OUT_OF_MEMORY if its allocations do.
    static constexpr size_t kLiveHeadroom = size_t(256) << 20;
    bool admits(size_t bytes, size_t liveFree) const
    {
        if (bytes + mReserved > mOpt.hbm_budget_bytes) return false;
        if (mInflight.empty() && mReserved == 0) return true;
        return bytes + kLiveHeadroom <= liveFree;
    }

    void dispatchLoop()
    {
        cudaSetDevice(mDevice);
        for (;;) {
            std::unique_lock<std::mutex> lk(mMu);
            Slot* slot = nullptr;
            size_t liveFree = 0;
            mCv.wait(lk, [&] {
                if (mStop) return true;
                if (mPending.empty()) return false;
                slot = freeSlot();
                if (slot == nullptr) return false;
                const size_t bytes = estimate(mPending.front()->n, 1);
                if (bytes + mReserved > mOpt.hbm_budget_bytes) return false;
                liveFree = (mInflight.empty() && mReserved == 0) ? ~size_t(0) : liveFreeBytes();
                return admits(bytes, liveFree);
            });
            if (mStop) {
                for (auto& r : mPending) finishLocked(*r, RBW_ERR_INVALID_ARG, "server stopped");
                mPending.clear();
                mDoneCv.notify_all();
                mCv.notify_all();
                return;
            }
            // form the batch: arrival order, within the slot limits and the memory budget
            uint64_t desc = 0;
            slot->reqs.clear();
            while (!mPending.empty() && slot->reqs.size() < mOpt.max_batch_queries) {
                const auto& r = mPending.front();
                if (desc + r->n > mOpt.max_batch_descriptors) break;
                if (!slot->reqs.empty() && !admits(estimate(desc + r->n, slot->reqs.size() + 1), liveFree)) break;
                desc += r->n;
                slot->reqs.push_back(r);
                mPending.pop_front();
            }
            const Clock::time_point formed = Clock::now();
            for (auto& r : slot->reqs) r->dispatched = formed;
            slot->reserved = estimate(desc, slot->reqs.size());
            mReserved += slot->reserved;
            mLiveFree = mLiveFree > slot->reserved ? mLiveFree - slot->reserved : 0;
            slot->busy = true;
            mBatches++;
            mBatchedRequests += slot->reqs.size();
            const uint32_t inflight = static_cast<uint32_t>(
                std::count_if(mSlots.begin(), mSlots.end(), [](const Slot& s) { return s.busy; }));
            mMaxInflight = std::max(mMaxInflight, inflight);
            lk.unlock();
            launch(*slot, desc);
            const Clock::time_point launched = Clock::now();
            lk.lock();
            for (auto& r : slot->reqs) r->launched = launched;
            mInflight.push_back(slot);
            mCv.notify_all();
        }
    }

    Slot* freeSlot()
    {
        for (Slot& s : mSlots)
            if (!s.busy) return &s;
        return nullptr;
    }

    // Copies the batch in, looks it up and scores it on the slot's stream (asynchronous).
    void launch(Slot& s, uint64_t desc)
    {
        s.status = RBW_OK;
        s.error.clear();
        const uint32_t nq = static_cast<uint32_t>(s.reqs.size());
        const uint32_t k = mOpt.max_results;
        uint64_t off = 0;
        for (uint32_t i = 0; i < nq; i++) {
            s.hOff[i] = off;
            off += s.reqs[i]->n;
        }
        s.hOff[nq] = off;
        void* dev = nullptr;
        const size_t descBytes = std::max<uint64_t>(desc, 1) * 128;
        const size_t leafBytes = (std::max<uint64_t>(desc, 1) * 4 + 7) & ~size_t(7);
        const size_t total = descBytes + leafBytes + (size_t(nq) + 1) * 8 + size_t(nq) * k * 8 + size_t(nq) * 4 + 256;
        try {
            RBW_CUDA(cudaMallocFromPoolAsync(&dev, total, libraryPool(), s.stream));
            uint8_t* dDesc = static_cast<uint8_t*>(dev);
            uint32_t* dLeaf = reinterpret_cast<uint32_t*>(dDesc + descBytes);
            uint64_t* dOff = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(dLeaf) + leafBytes);
            uint32_t* dDocs = reinterpret_cast<uint32_t*>(dOff + nq + 1);
            float* dScores = reinterpret_cast<float*>(dDocs + size_t(nq) * k);
            uint32_t* dCount = reinterpret_cast<uint32_t*>(dScores + size_t(nq) * k);
            for (uint32_t i = 0; i < nq; i++) {
                const Request& r = *s.reqs[i];
                if (r.n)
                    RBW_CUDA(cudaMemcpyAsync(dDesc + s.hOff[i] * 128, r.desc, size_t(r.n) * 128,
                                             cudaMemcpyHostToDevice, s.stream));
            }
            RBW_CUDA(cudaMemcpyAsync(dOff, s.hOff, (size_t(nq) + 1) * 8, cudaMemcpyHostToDevice, s.stream));
            uint32_t kernels = 0;
            int rc = desc ? rbw_voc_lookup_ex(mVoc, dDesc, desc, dLeaf, RBW_LOOKUP_AUTO, s.stream, &kernels) : RBW_OK;
            if (rc != RBW_OK) throw Error(static_cast<Status>(rc), rbw_last_error());
            rc = rbw_db_query_batched_host_offsets(mDb, dLeaf, dOff, s.hOff, nq, k, dDocs, dScores, dCount, s.stream);
            if (rc != RBW_OK) throw Error(static_cast<Status>(rc), rbw_last_error());
            RBW_CUDA(cudaMemcpyAsync(s.hDocs, dDocs, size_t(nq) * k * 4, cudaMemcpyDeviceToHost, s.stream));
            RBW_CUDA(cudaMemcpyAsync(s.hScores, dScores, size_t(nq) * k * 4, cudaMemcpyDeviceToHost, s.stream));
            RBW_CUDA(cudaMemcpyAsync(s.hCount, dCount, size_t(nq) * 4, cudaMemcpyDeviceToHost, s.stream));
            RBW_CUDA(cudaFreeAsync(dev, s.stream));
            dev = nullptr;
        } catch (const Error& e) {
            s.status = e.status;
            s.error = e.what();
        } catch (const std::exception& e) {
            s.status = RBW_ERR_INTERNAL;
            s.error = e.what();
        }
        if (dev) cudaFreeAsync(dev, s.stream);
        cudaEventRecord(s.done, s.stream);
    }

    void completeLoop()
    {
        cudaSetDevice(mDevice);
        for (;;) {
            Slot* s = nullptr;
            {
                std::unique_lock<std::mutex> lk(mMu);
                mCv.wait(lk, [&] { return !mInflight.empty() || (mStop && mPending.empty()); });
                if (mInflight.empty()) return;
                s = mInflight.front();
            }
            const cudaError_t e = cudaEventSynchronize(s->done);
            std::lock_guard<std::mutex> lk(mMu);
            mInflight.pop_front();
            const uint32_t k = mOpt.max_results;
            for (size_t i = 0; i < s->reqs.size(); i++) {
                Request& r = *s->reqs[i];
                if (s->status != RBW_OK || e != cudaSuccess) {
                    finishLocked(r, s->status != RBW_OK ? s->status : RBW_ERR_CUDA,
                                 s->status != RBW_OK ? s->error : cudaGetErrorString(e));
                    continue;
                }
                const uint32_t n = std::min(s->hCount[i], k);
                r.docs.assign(s->hDocs + i * k, s->hDocs + i * k + n);
                r.scores.assign(s->hScores + i * k, s->hScores + i * k + n);
                finishLocked(r, RBW_OK, "");
            }
            s->reqs.clear();
            mReserved -= s->reserved;
            s->reserved = 0;
            s->busy = false;
            mDoneCv.notify_all();
            mCv.notify_all();
        }
    }

    void finishLocked(Request& r, int status, const std::string& err)
    {
        r.status = status;
        r.error = err;
        r.finished = Clock::now();
        r.done = true;
        // the batch that copied these descriptors has completed (or never ran)
        mPinned.give(r.desc, r.descClass);
        r.desc = nullptr;
        if (status == RBW_OK) {
            auto ms = [](Clock::time_point a, Clock::time_point b) {
                return std::chrono::duration<double, std::milli>(b - a).count();
            };
            mLatencies.push_back(ms(r.submitted, r.finished));
            mStage[0].push_back(ms(r.submitted, r.dispatched));
            mStage[1].push_back(ms(r.dispatched, r.launched));
            mStage[2].push_back(ms(r.launched, r.finished));
        }
    }

    PinnedPool mPinned; // destroyed after the threads (declared before them)
    size_t mLiveFree = 0;
    Clock::time_point mLiveAt{};
    const rbw_vocabulary* mVoc;
    rbw_database* mDb;
    rbw_server_options mOpt;
    int mDevice = 0;
    uint32_t mLevels = 0;
    std::vector<Slot> mSlots;
    std::deque<std::shared_ptr<Request>> mPending;
    std::deque<Slot*> mInflight;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> mAll;
    std::vector<double> mLatencies;
    std::vector<double> mStage[3]; // queue, launch, device (ms), as mLatencies
    uint64_t mNextId = 0, mSubmitted = 0, mBatches = 0, mBatchedRequests = 0;
    uint32_t mMaxInflight = 0;
    size_t mReserved = 0;
    bool mStop = false;
    std::mutex mMu;
    std::condition_variable mCv, mDoneCv;
    std::thread mDispatcher, mCompleter;
};

} // namespace
} // namespace rbw

struct rbw_server {
    std::unique_ptr<rbw::Server> s;
};

namespace {
rbw::Server& serverOf(rbw_server* h)
{
    if (h == nullptr || !h->s) throw rbw::Error(rbw::kInvalidArg, "null server handle");
    return *h->s;
}
} // namespace

extern "C" {

void rbw_server_options_default(rbw_server_options* o)
{
    if (o == nullptr) return;
    o->max_batch_queries = 256;
    o->max_batch_descriptors = 1u << 21;
    o->max_inflight_batches = 3;
    o->max_results = 100;
    o->hbm_budget_bytes = 0;
}

int rbw_server_create(const rbw_vocabulary* voc, rbw_database* db, const rbw_server_options* opts, rbw_server** out)
{
    return rbw::runGuarded([&] {
        if (out == nullptr || db == nullptr) throw rbw::Error(rbw::kInvalidArg, "null argument");
        *out = nullptr;
        rbw_server_options o;
        rbw_server_options_default(&o);
        if (opts) o = *opts;
        *out = new rbw_server{std::make_unique<rbw::Server>(voc, db, o)};
    });
}

void rbw_server_destroy(rbw_server* s) { delete s; }

int rbw_server_submit(rbw_server* s, const void* host_desc, uint32_t n_desc, uint64_t* request_id)
{
    return rbw::runGuarded([&] {
        if (request_id == nullptr) throw rbw::Error(rbw::kInvalidArg, "null request id");
        *request_id = serverOf(s).submit(static_cast<const uint8_t*>(host_desc), n_desc);
    });
}

int rbw_server_wait(rbw_server* s, uint64_t request_id, int64_t timeout_us, uint32_t* docs, float* scores,
                    uint32_t capacity, uint32_t* n_out, double* latency_ms)
{
    return rbw::runGuarded([&] {
        if (!serverOf(s).wait(request_id, timeout_us, docs, scores, capacity, n_out, latency_ms))
            throw rbw::Error(rbw::kTimeout, "request not finished within the timeout");
    });
}

int rbw_server_get_stats(rbw_server* s, rbw_server_stats* stats)
{
    return rbw::runGuarded([&] {
        if (stats == nullptr) throw rbw::Error(rbw::kInvalidArg, "null stats");
        serverOf(s).stats(stats);
    });
}

int rbw_server_batch_bytes(rbw_server* s, uint64_t n_desc, uint32_t n_requests, uint64_t* bytes)
{
    return rbw::runGuarded([&] {
        if (bytes == nullptr) throw rbw::Error(rbw::kInvalidArg, "null output");
        *bytes = serverOf(s).batchBytes(n_desc, n_requests);
    });
}

int rbw_server_reset_stats(rbw_server* s)
{
    return rbw::runGuarded([&] { serverOf(s).resetStats(); });
}

} // extern "C"
