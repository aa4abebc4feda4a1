// Allocation-free variant of the 32-bit-key radix sort.
//
// Some callers cannot call cudaMalloc: a host application that owns every
// byte of device memory through its own pool and forbids libraries from
// allocating behind its back, or a caller on a latency-critical path where
// the implicit device-wide synchronisation of cudaMalloc/cudaFree is not
// acceptable.  This entry point sorts with scratch that lives in a
// file-scope device array instead of caller- or library-allocated memory.
//
// Limits and sharing rules:
//   - at most kNoAllocMaxPairs (1,048,576) key/value pairs per call; the
//     array costs 8.5 MiB (8,912,896 bytes) on every device that loads the
//     library and stays resident until the process exits;
//   - every call uses the same array: calls that overlap on the GPU (on
//     different streams, or from different host threads) race and corrupt
//     each other; serialise them on one stream;
//   - the array keeps the previous call's contents; the sort clears the
//     parts that must start at zero (histograms, tile tickets, tile status,
//     error word) itself before using them;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make
//     that first call before any stream capture.  The cached address is
//     kept for the life of the process, so do not call this entry point on
//     a device after cudaDeviceReset (or any other teardown of its primary
//     context): the module, and with it the array, is loaded anew there;
//   - a look-back wait of the sort that gives up (bounded, and not expected
//     in practice: it takes a tile stalled for millions of polls) sets an
//     error word inside the array, which this entry point cannot return
//     without a device synchronisation; the order of that call's output is
//     then undefined and nothing reports it.
#include <mutex>

#include "../../include/mrb200.h"
#include "common.cuh"
#include "sort.cuh"

namespace mrb {
namespace {

constexpr uint32_t kNoAllocMaxPairs = 1u << 20;
// radix_sort_temp_bytes(kNoAllocMaxPairs, 4, 0, 32) rounded up
constexpr size_t kNoAllocBytes = 8704u * 1024u;

__device__ __align__(256) unsigned char g_sort_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

int scratch_for_current_device(void** out) {
    int dev = 0;
    MRB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("no-alloc sort: device %d out of the supported range", dev);
        return MRB_E_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || !p) {
            set_error("no-alloc sort: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return MRB_E_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return 0;
}

}  // namespace
}  // namespace mrb

extern "C" int mrb_radix_sort_pairs_u32_noalloc(uint32_t* keys, uint32_t* vals, uint32_t n,
                                                int beginBit, int endBit, int descending,
                                                void* stream) {
    using namespace mrb;
    if (beginBit < 0 || endBit > 32 || beginBit > endBit) {
        set_error("bit range [%d, %d) invalid for 32-bit keys", beginBit, endBit);
        return MRB_E_ARG;
    }
    if (n > kNoAllocMaxPairs) {
        set_error("no-alloc sort: %u pairs exceed the maximum of %u", n, kNoAllocMaxPairs);
        return MRB_E_ARG;
    }
    if (n == 0) return 0;
    const size_t need = radix_sort_temp_bytes(n, 4, beginBit, endBit);
    if (need > kNoAllocBytes) {
        set_error("no-alloc sort: %zu scratch bytes needed, %zu available", need, kNoAllocBytes);
        return MRB_E_ARG;
    }
    void* scratch = nullptr;
    int r = scratch_for_current_device(&scratch);
    if (r) return r;
    return radix_sort_pairs<uint32_t>(keys, vals, nullptr, n, beginBit, endBit, descending != 0,
                                      scratch, kNoAllocBytes, static_cast<cudaStream_t>(stream),
                                      false);
}
