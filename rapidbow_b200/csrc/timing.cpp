#include "timing.h"
#include "rbw_common.cuh"

#include <atomic>
#include <mutex>
#include <vector>

namespace rbw {
namespace {

struct Record {
    TimedKernel kernel;
    cudaEvent_t start;
    cudaEvent_t stop;
};

std::atomic<bool> gEnabled{false};
std::mutex gMu;
std::vector<Record> gRecords;
std::vector<cudaEvent_t> gPool;

cudaEvent_t takeEvent()
{
    if (!gPool.empty()) {
        cudaEvent_t e = gPool.back();
        gPool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    RBW_CUDA(cudaEventCreate(&e));
    return e;
}

} // namespace

bool timingEnabled() { return gEnabled.load(std::memory_order_relaxed); }

void timingEnable(bool on) { gEnabled.store(on); }

void timingReset()
{
    std::lock_guard<std::mutex> lk(gMu);
    for (auto& r : gRecords) {
        gPool.push_back(r.start);
        gPool.push_back(r.stop);
    }
    gRecords.clear();
}

void timingRead(TimedKernel k, double* totalMs, uint64_t* launches)
{
    std::lock_guard<std::mutex> lk(gMu);
    double total = 0;
    uint64_t n = 0;
    for (const auto& r : gRecords) {
        if (r.kernel != k) continue;
        float ms = 0;
        RBW_CUDA(cudaEventElapsedTime(&ms, r.start, r.stop));
        total += ms;
        n++;
    }
    if (totalMs) *totalMs = total;
    if (launches) *launches = n;
}

ScopedKernelTimer::ScopedKernelTimer(TimedKernel k, cudaStream_t s) : mKernel{k}, mStream{s}
{
    if (!timingEnabled()) return;
    std::lock_guard<std::mutex> lk(gMu);
    mStart = takeEvent();
    RBW_CUDA(cudaEventRecord(mStart, mStream));
    mActive = true;
}

ScopedKernelTimer::~ScopedKernelTimer()
{
    if (!mActive) return;
    std::lock_guard<std::mutex> lk(gMu);
    cudaEvent_t stop = nullptr;
    try {
        stop = takeEvent();
    } catch (...) {
        gPool.push_back(mStart);
        return;
    }
    if (cudaEventRecord(stop, mStream) != cudaSuccess) {
        gPool.push_back(mStart);
        gPool.push_back(stop);
        return;
    }
    gRecords.push_back(Record{mKernel, mStart, stop});
}

} // namespace rbw
