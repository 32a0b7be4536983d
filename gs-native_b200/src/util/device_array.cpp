// Allocation hook of the stage classes (see device_array.h).
#include "util/device_array.h"

#include <atomic>

namespace gs_native {

namespace {
std::atomic<DeviceAllocFn> g_alloc_hook{nullptr};
}  // namespace

void SetDeviceAllocHook(DeviceAllocFn fn) { g_alloc_hook.store(fn); }

cudaError_t DeviceAlloc(void** ptr, size_t bytes) {
    DeviceAllocFn fn = g_alloc_hook.load();
    if (fn) return fn(ptr, bytes);
    return cudaMalloc(ptr, bytes);
}

}  // namespace gs_native
