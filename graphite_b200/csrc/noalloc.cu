// gbReduceSumNoAlloc: the deterministic float64 sum of FvmFieldReduceSum for
// callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a
// reduction: hosts that hand out all device memory from their own pool and
// forbid other allocations, and plugins that must keep their device footprint
// fixed after setup.  The mesh/field entry points allocate their
// scratch (reduction partials, gradients) on first use; this entry point
// allocates nothing.  Its scratch -- one float64 partial sum per block of
// 2048 inputs -- lives in the file-scope array below, which every GPU that
// loads the library holds until the process exits.
#include <mutex>
#include <string>

#include "gb_device.cuh"
#include "gb_internal.h"

namespace gb {
namespace {

// Partial sums: at most this many blocks of kNoAllocBlockItems inputs.
constexpr int kNoAllocPartials = 4096;                           // 32 KiB per GPU
constexpr int64_t kNoAllocBlockItems = (int64_t)kBlock * 8;      // inputs per block
constexpr int64_t kNoAllocMaxItems = (int64_t)kNoAllocPartials * kNoAllocBlockItems;   // 8,388,608
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

// Device address of g_noalloc_partials, resolved once per device.  In host
// code the array's name is only a host-side stand-in for the symbol, so the
// kernels are given this address.  The cached address belongs to the
// device's current context: after cudaDeviceReset the module may load at
// another address, so a caller that resets a device must not use this entry
// point on it again in the same process.
std::mutex g_mu;
double* g_ptr[kMaxDevices] = {nullptr};

bool scratch_for_current_device(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("gbReduceSumNoAlloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return false;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("gbReduceSumNoAlloc: device ordinal out of range");
        return false;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p) {
            set_error(std::string("gbReduceSumNoAlloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return false;
        }
        g_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_ptr[dev];
    return true;
}

// Whether p is device (or managed) memory this context can write: a host
// pointer given here would be written through by the kernel.
bool device_pointer(const void* p) {
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();   // the error is not sticky; clear it so later calls do not see it
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" int gbReduceSumNoAlloc(const float* values, uint64_t n, double* result, void* stream) {
    clear_error();
    if (!values || !result || !device_pointer(values) || !device_pointer(result)) {
        set_error("gbReduceSumNoAlloc: values and result must be device (or managed) memory");
        return 1;
    }
    if (n > (uint64_t)kNoAllocMaxItems) {
        set_error("gbReduceSumNoAlloc: " + std::to_string(n) + " values exceed the maximum of " +
                  std::to_string(kNoAllocMaxItems) + " (" + std::to_string(kNoAllocPartials) +
                  " partial sums of " + std::to_string(kNoAllocBlockItems) + " values)");
        return 1;
    }
    double* partials = nullptr;
    if (!scratch_for_current_device(&partials)) return 1;
    cudaStream_t s = (cudaStream_t)stream;
    const int blocks = n == 0 ? 1 : (int)((n + kNoAllocBlockItems - 1) / kNoAllocBlockItems);
    // every partial that stage 2 reads is written by stage 1 of this call,
    // so nothing left from an earlier call needs clearing
    launch_reduce_partials_blocks((int64_t)n, values, partials, blocks, s);
    launch_reduce_final(blocks, partials, result, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("gbReduceSumNoAlloc: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}
