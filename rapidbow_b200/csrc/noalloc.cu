// Lookup that allocates nothing.
//
// Some callers cannot allocate device memory when they look descriptors up: real-time or
// serving loops that must not hit the driver allocator (cudaMalloc can synchronise the device
// and its latency is unbounded), plug-ins running inside a host application that owns all GPU
// memory, and hosts that hand this library a fixed memory budget up front.  For them,
// rbw_voc_lookup_noalloc runs the same tensor-core lookup as rbw_voc_lookup, but its working
// memory (the regroup permutation, histograms and tile lists between passes) lives in one
// file-scope device array of kNoAllocScratchBytes, reserved on every GPU that loads this
// library for the life of the process.
//
// Rules for callers:
//   * the first call on a device looks the array's device address up (cudaGetSymbolAddress)
//     with that device current; make that first call before any stream capture begins.  The
//     address is kept for the life of the process: after cudaDeviceReset on that device the
//     module is loaded again and the kept address is stale, so the entry point must not be used
//     after a device reset;
//   * all calls on a device share the one array: calls whose kernels may overlap on the GPU
//     (different streams without ordering between them, or several host threads) race on it
//     and must be serialised by the caller;
//   * the array keeps whatever the previous call left in it; the lookup clears the parts it
//     needs zeroed (histograms and cursors) itself on the stream;
//   * a call whose descriptors need more working memory than the array holds is rejected with
//     RBW_ERR_INVALID_ARG before anything is launched (rbw_voc_lookup_scratch_bytes reports
//     the need; about one million descriptors per call fit for a 4-level, 16-ary tree).
#include "capi_internal.h"

#include <mutex>
#include <string>

namespace rbw {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20; // 8 MiB

static __device__ __align__(256) unsigned char gNoAllocScratch[kNoAllocScratchBytes];

// Device address of gNoAllocScratch, looked up once per device with that device current.
void* noAllocScratchAddress()
{
    static std::mutex mu;
    static void* addr[kMaxDevices] = {};
    const int dev = currentDevice();
    std::lock_guard<std::mutex> lk(mu);
    if (addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, gNoAllocScratch);
        if (e != cudaSuccess || p == nullptr) {
            throw Error(kCudaError, std::string("cudaGetSymbolAddress of the lookup scratch array failed: ") +
                                        cudaGetErrorString(e));
        }
        addr[dev] = p;
    }
    return addr[dev];
}

} // namespace
} // namespace rbw

extern "C" int rbw_voc_lookup_noalloc(const rbw_vocabulary* voc, const void* dev_desc, uint32_t nb_desc,
                                      uint32_t* dev_leaf, void* stream)
{
    return rbw::runGuarded([&] {
        const rbw::Vocabulary& v = rbw::vocabularyOf(voc);
        if (v.floatCenters())
            throw rbw::Error(rbw::kUnsupported, "rbw_voc_lookup_noalloc: float-center vocabularies are not supported");
        const size_t need = rbw::lookupScratchBytes(v.branch(), v.levels(), nb_desc);
        if (need > rbw::kNoAllocScratchBytes) {
            throw rbw::Error(rbw::kInvalidArg,
                             "rbw_voc_lookup_noalloc: " + std::to_string(nb_desc) + " descriptors need " +
                                 std::to_string(need) + " bytes of working memory, more than its fixed " +
                                 std::to_string(rbw::kNoAllocScratchBytes) + "-byte array; split the call");
        }
        void* scratch = rbw::noAllocScratchAddress();
        v.lookup(static_cast<const uint8_t*>(dev_desc), nb_desc, dev_leaf, rbw::kLookupTensorU8,
                 static_cast<cudaStream_t>(stream), scratch, rbw::kNoAllocScratchBytes);
    });
}
