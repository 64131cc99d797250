// Shared device/host helpers for the RapidBoW-B200 kernels (sm_100a only).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "RapidBoW-B200 kernels target sm_100a only"
#endif

namespace rbw {

constexpr uint32_t kDims = 128;          // SIFT descriptor bytes (RapidBoW.h:50)
constexpr uint32_t kMaxBranch = 16;      // centers per node slot in device layouts
constexpr uint32_t kInvalidIdx = 0xFFFFFFFFu;
constexpr int32_t kPadNorm = 0x3FFFFFFF; // |c|^2 of padding centers: never the argmin

// Error codes shared with the C ABI (include/rapidbow_b200.h).
enum Status : int {
    kOk = 0,
    kInvalidArg = 1,
    kUnsupported = 2,
    kOutOfMemory = 3,
    kCudaError = 4,
    kTimeout = 5,
    kInvalidBlob = 6,
    kDuplicate = 7,
    kInternal = 8,
};

struct Error : std::runtime_error {
    Status status;
    Error(Status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void cudaThrow(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        const Status s = (e == cudaErrorMemoryAllocation) ? kOutOfMemory : kCudaError;
        throw Error(s, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    }
}
#define RBW_CUDA(call) ::rbw::cudaThrow((call), #call)

inline uint64_t levelBeg(uint32_t B, uint32_t level)
{
    uint64_t acc = 0;
    for (uint32_t i = 0; i < level; i++) acc = acc * B + 1;
    return acc;
}
inline uint64_t ipow(uint64_t b, uint32_t e)
{
    uint64_t r = 1;
    while (e--) r *= b;
    return r;
}
template <typename T>
__host__ __device__ constexpr T ceilDiv(T a, T b) { return (a + b - 1) / b; }

constexpr int kMaxDevices = 64;

// Ordinal of the calling thread's current device.  Per-device state (function attributes, SM
// counts, pools) is keyed by it: attributes such as the dynamic shared-memory limit belong to
// one device's context and must be set again for every other device the process uses.
inline int currentDevice()
{
    int dev = 0;
    RBW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(kUnsupported, "device ordinal out of range");
    return dev;
}

// Number of SMs of the current device.
inline int currentSmCount()
{
    static std::atomic<int> sms[kMaxDevices] = {};
    const int dev = currentDevice();
    int v = sms[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        RBW_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        sms[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// Sets a kernel's dynamic shared-memory limit once per device (idempotent, so a race between
// two threads only sets it twice).
inline void setMaxDynamicSmemOncePerDevice(const void* kernel, int bytes, std::atomic<uint64_t>& doneMask)
{
    const int dev = currentDevice();
    const uint64_t bit = uint64_t(1) << dev;
    if (doneMask.load(std::memory_order_acquire) & bit) return;
    RBW_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    doneMask.fetch_or(bit, std::memory_order_acq_rel);
}

// Device-side error record written by bounded waits and bounds checks.
struct DeviceErrors {
    uint32_t code;      // 0 = none, 1 = wait timeout, 2 = bounds
    uint32_t where;     // site id
    uint32_t block;
    uint32_t detail;
};

#ifdef __CUDACC__
// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smemAddr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globalTimerNs()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbarInit(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fenceMbarInit()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbarArriveExpectTx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbarArrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}
// One bounded try: the thread is suspended (not spinning) until the phase completes or the
// hint (ns) expires, so waiting warps leave the issue slots to the warps doing work.
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, uint32_t parity, uint32_t suspendNs = 1000000u)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity), "r"(suspendNs)
        : "memory");
    return ok != 0;
}

constexpr uint64_t kWaitLimitNs = 2000000000ull; // 2 s: far above any legitimate wait

// Bounded wait on an mbarrier phase.  On timeout (or when another warp already aborted) it
// records the site in `err`, raises the CTA-wide abort flag and returns false; the caller
// then stops issuing work and falls through to the kernel's teardown.
__device__ __forceinline__ bool mbarWait(uint64_t* bar, uint32_t parity, volatile uint32_t* abortFlag,
                                         DeviceErrors* err, uint32_t site)
{
    if (mbarTryWait(bar, parity)) return true;
    const uint64_t t0 = globalTimerNs();
    for (;;) {
        if (mbarTryWait(bar, parity)) return true;
        if (*abortFlag) return false;
        if (globalTimerNs() - t0 > kWaitLimitNs) {
            *abortFlag = 1;
            if (err != nullptr && atomicCAS(&err->code, 0u, 1u) == 0u) {
                err->where = site;
                err->block = blockIdx.x;
                err->detail = parity;
            }
            return false;
        }
    }
}

// 4-byte asynchronous global -> shared copy (no register dependency) and its group fences.
__device__ __forceinline__ void cpAsync4(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smemAddr(dst)), "l"(src) : "memory");
}
// 16-byte asynchronous global -> shared copy, cached in L2 only.
__device__ __forceinline__ void cpAsync16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smemAddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// TMA: 2D tiled load.
__device__ __forceinline__ void tmaLoad2d(void* dst, const CUtensorMap* map, int32_t x, int32_t y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smemAddr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smemAddr(bar))
        : "memory");
}
// Untiled bulk copy global -> shared (16-B aligned addresses, size multiple of 16).
__device__ __forceinline__ void bulkLoad(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smemAddr(dst)),
        "l"(src), "r"(bytes), "r"(smemAddr(bar))
        : "memory");
}

// tcgen05 (5th-generation tensor core, accumulators in tensor memory)
__device__ __forceinline__ void tmemAlloc(uint32_t* dstSmem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(dstSmem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmemRelinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmemDealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, uint8 x uint8 -> int32, M = 128, N from idesc.
__device__ __forceinline__ void mmaU8(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc,
                                      uint32_t accumulate)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, bf16 x bf16 -> fp32, M = 128, N from idesc.
__device__ __forceinline__ void mmaBf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc,
                                        uint32_t accumulate)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dTmem),
        "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
// Arrive (once) on `bar` when all previously issued MMAs of this thread have completed.
__device__ __forceinline__ void mmaCommit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smemAddr(bar))
                 : "memory");
}

// 32 lanes x 16 columns of 32-bit accumulators; thread i gets lane (base + i).
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
// Waits until the tcgen05.ld results are in registers; the operands tie the 16 registers to
// the wait so no use of them is scheduled before it.
__device__ __forceinline__ void tmemWaitTie(uint32_t (&r)[16])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                   "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]),
                   "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
}

// Shared-memory matrix descriptor for a K-major operand laid out in 128-byte swizzle atoms
// (8 rows x 128 B, atoms stacked densely along M/N): SBO = 1024 B, LBO = 16 B (unused),
// descriptor version 1, layout type 2 (SWIZZLE_128B).  `addr` is the shared address of the
// first row of the slice, advanced by k*bytesPerK inside the atom for the K steps.
__device__ __forceinline__ uint64_t smemDescSw128(uint32_t addr)
{
    uint64_t d = 0;
    d |= uint64_t((addr >> 4) & 0x3FFFu);
    d |= uint64_t(1u) << 16;              // LBO (16 B units)
    d |= uint64_t(1024u >> 4) << 32;      // SBO (16 B units)
    d |= uint64_t(1u) << 46;              // version
    d |= uint64_t(2u) << 61;              // SWIZZLE_128B
    return d;
}

// Instruction descriptor (M = 128, K-major A and B, uint8 x uint8 -> s32).
__host__ __device__ constexpr uint32_t idescU8(uint32_t n)
{
    return (2u << 4)              // D = S32
           | (0u << 7)            // A = UINT8
           | (0u << 10)           // B = UINT8
           | ((n >> 3) << 17)     // N
           | ((128u >> 4) << 24); // M
}

// Instruction descriptor (M = 128, K-major A and B, bf16 x bf16 -> fp32).
__host__ __device__ constexpr uint32_t idescBf16(uint32_t n)
{
    return (1u << 4)              // D = F32
           | (1u << 7)            // A = BF16
           | (1u << 10)           // B = BF16
           | ((n >> 3) << 17)     // N
           | ((128u >> 4) << 24); // M
}

#endif // __CUDACC__

} // namespace rbw
