// Test infrastructure only: a minimal stand-in for the external `cuda-utils` helper library
// that the reference sources include (`#include <cuda_utils.h>`) but that the reference does
// not vendor (its CMakeLists.txt:13-14,26 point at a sibling checkout).  This header lets the
// UNMODIFIED reference sources compile into oracle/_ref/ so the reference itself can serve as
// a checker.  Nothing in the product links against this file.
//
// Only the symbols the reference uses are provided, each written from its use sites:
//   CudaMemType, CudaMem<T,type>, allocCudaMem<T,type,zero>, cudaCheck, divUp, roundUp,
//   lane_id, unused, CudaHostAllocator, CudaManagedAllocator, makeScopeGuard, getCudaDevice,
//   DirectMappingHash.   (VectorMap.h and CudaEventPool.h hold the other two.)
#pragma once
#include <cuda_runtime_api.h>
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

inline void cudaCheck(cudaError_t err)
{
    if (err != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorName(err) + ": " +
                                 cudaGetErrorString(err));
    }
}

template <typename A, typename B>
__host__ __device__ constexpr auto divUp(A a, B b) -> std::common_type_t<A, B>
{
    return (a + b - 1) / b;
}

template <typename A, typename B>
__host__ __device__ constexpr auto roundUp(A a, B b) -> std::common_type_t<A, B>
{
    return divUp(a, b) * b;
}

template <typename... Args>
__host__ __device__ inline void unused(Args&&...) {}

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t lane_id()
{
    uint32_t id;
    asm("mov.u32 %0, %%laneid;" : "=r"(id));
    return id;
}
#endif

enum class CudaMemType { kDevice, kPinned, kManaged };

namespace shim_detail {
template <CudaMemType type>
struct CudaDeleter {
    void operator()(void* p) const
    {
        if (p == nullptr) return;
        if (type == CudaMemType::kPinned) {
            cudaFreeHost(p);
        } else {
            cudaFree(p);
        }
    }
};
} // namespace shim_detail

// Owning pointer to CUDA memory with element access (used as `mem[i]`, `mem.get()`,
// `mem.release()`, `mem.reset()`, and constructed from a raw pointer).
template <typename T, CudaMemType type = CudaMemType::kDevice>
class CudaMem : public std::unique_ptr<T[], shim_detail::CudaDeleter<type>>
{
    using Base = std::unique_ptr<T[], shim_detail::CudaDeleter<type>>;

public:
    CudaMem() = default;
    explicit CudaMem(T* p) : Base{p} {}
    CudaMem(CudaMem&&) noexcept = default;
    CudaMem& operator=(CudaMem&&) noexcept = default;
};

template <typename T, CudaMemType type = CudaMemType::kDevice, bool zero = false>
CudaMem<T, type> allocCudaMem(size_t nbElems)
{
    void* p = nullptr;
    const size_t bytes = sizeof(T) * nbElems;
    if (bytes != 0) {
        switch (type) {
        case CudaMemType::kDevice: cudaCheck(cudaMalloc(&p, bytes)); break;
        case CudaMemType::kPinned: cudaCheck(cudaMallocHost(&p, bytes)); break;
        case CudaMemType::kManaged: cudaCheck(cudaMallocManaged(&p, bytes)); break;
        }
        if (zero) {
            if (type == CudaMemType::kPinned) {
                std::memset(p, 0, bytes);
            } else {
                cudaCheck(cudaMemset(p, 0, bytes));
            }
        }
    }
    return CudaMem<T, type>{static_cast<T*>(p)};
}

template <typename T, CudaMemType type>
struct CudaAllocatorBase {
    using value_type = T;
    CudaAllocatorBase() = default;
    template <typename U>
    CudaAllocatorBase(const CudaAllocatorBase<U, type>&) {}
    T* allocate(size_t n)
    {
        void* p = nullptr;
        if (type == CudaMemType::kPinned) {
            cudaCheck(cudaMallocHost(&p, sizeof(T) * n));
        } else {
            cudaCheck(cudaMallocManaged(&p, sizeof(T) * n));
        }
        return static_cast<T*>(p);
    }
    void deallocate(T* p, size_t)
    {
        if (type == CudaMemType::kPinned) {
            cudaFreeHost(p);
        } else {
            cudaFree(p);
        }
    }
    template <typename U>
    bool operator==(const CudaAllocatorBase<U, type>&) const { return true; }
    template <typename U>
    bool operator!=(const CudaAllocatorBase<U, type>&) const { return false; }
};

template <typename T>
struct CudaHostAllocator : CudaAllocatorBase<T, CudaMemType::kPinned> {
    template <typename U>
    struct rebind { using other = CudaHostAllocator<U>; };
    CudaHostAllocator() = default;
    template <typename U>
    CudaHostAllocator(const CudaHostAllocator<U>&) {}
};

template <typename T>
struct CudaManagedAllocator : CudaAllocatorBase<T, CudaMemType::kManaged> {
    template <typename U>
    struct rebind { using other = CudaManagedAllocator<U>; };
    CudaManagedAllocator() = default;
    template <typename U>
    CudaManagedAllocator(const CudaManagedAllocator<U>&) {}
};

template <typename F>
class ScopeGuard
{
public:
    explicit ScopeGuard(F f) : mF{std::move(f)} {}
    ScopeGuard(ScopeGuard&& o) noexcept : mF{std::move(o.mF)}, mActive{o.mActive} { o.mActive = false; }
    ~ScopeGuard()
    {
        if (mActive) mF();
    }

private:
    F mF;
    bool mActive{true};
};

template <typename F>
ScopeGuard<F> makeScopeGuard(F f)
{
    return ScopeGuard<F>{std::move(f)};
}

inline int getCudaDevice()
{
    int dev = 0;
    cudaCheck(cudaGetDevice(&dev));
    return dev;
}

// Identity hash for small integer keys.
template <typename T>
struct DirectMappingHash {
    size_t operator()(const T& v) const noexcept { return static_cast<size_t>(v); }
};
