// Grow-only device allocations used by the stage classes. Growth never
// preserves contents (callers that need it copy explicitly); a failed growth
// leaves the previous allocation untouched so the owning object stays usable,
// which is the rollback behaviour of the reference's stage classes
// (renderer.cu:383-429).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <utility>

namespace gs_native {

// Optional allocation hook so tests can inject cudaMalloc failures on the host.
using DeviceAllocFn = cudaError_t (*)(void** ptr, size_t bytes);
void SetDeviceAllocHook(DeviceAllocFn fn);
cudaError_t DeviceAlloc(void** ptr, size_t bytes);

template <typename T>
class DeviceArray {
public:
    DeviceArray() = default;
    ~DeviceArray() { cudaFree(data_); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    DeviceArray(DeviceArray&& o) noexcept : data_(o.data_), capacity_(o.capacity_) {
        o.data_ = nullptr;
        o.capacity_ = 0;
    }
    DeviceArray& operator=(DeviceArray&& o) noexcept {
        std::swap(data_, o.data_);
        std::swap(capacity_, o.capacity_);
        return *this;
    }

    // Ensures room for `count` elements; returns false (and keeps the old buffer)
    // when the allocation fails.
    bool Reserve(size_t count) {
        if (count <= capacity_ && data_) return true;
        void* p = nullptr;
        if (DeviceAlloc(&p, (count ? count : 1) * sizeof(T)) != cudaSuccess) return false;
        cudaFree(data_);
        data_ = static_cast<T*>(p);
        capacity_ = count;
        return true;
    }
    void Reset() {
        cudaFree(data_);
        data_ = nullptr;
        capacity_ = 0;
    }
    T* get() const { return data_; }
    size_t capacity() const { return capacity_; }

private:
    T* data_ = nullptr;
    size_t capacity_ = 0;
};

}  // namespace gs_native
