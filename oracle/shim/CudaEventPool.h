// Test infrastructure only: stand-in for the external `CudaEventPool.h` used by the reference's
// DeviceKernelArg.h:26,83 (`cudapp::PooledCudaEvent`, `cudapp::createPooledCudaEvent()`,
// `event.get()`).  A plain RAII event is enough for those uses.
#pragma once
#include "cuda_utils.h"

namespace cudapp {
class PooledCudaEvent
{
public:
    PooledCudaEvent() = default;
    explicit PooledCudaEvent(cudaEvent_t ev) : mEvent{ev} {}
    PooledCudaEvent(PooledCudaEvent&& o) noexcept : mEvent{o.mEvent} { o.mEvent = nullptr; }
    PooledCudaEvent& operator=(PooledCudaEvent&& o) noexcept
    {
        std::swap(mEvent, o.mEvent);
        return *this;
    }
    ~PooledCudaEvent()
    {
        if (mEvent != nullptr) cudaEventDestroy(mEvent);
    }
    cudaEvent_t get() const { return mEvent; }

private:
    cudaEvent_t mEvent{nullptr};
};

inline PooledCudaEvent createPooledCudaEvent()
{
    cudaEvent_t ev = nullptr;
    cudaCheck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    return PooledCudaEvent{ev};
}
} // namespace cudapp
