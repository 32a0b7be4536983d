// Spatial (Morton) reordering of a parameter block (gs-native extension; the
// reference keeps the order its density step writes, density_controller.cu:
// 168-243). The permutation changes no rendered or trained value; it gives the
// Gaussians of one view long id runs, which a visibility-masked Adam step turns
// into skipped HBM sectors.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "core/types/buffers.h"
#include "util/device_array.h"

namespace gs_native {

class SpatialOrder {
public:
    void SetStream(cudaStream_t stream) { stream_ = stream; }
    // Permutation perm (device, count entries): new Gaussian i is old perm[i],
    // in ascending Morton order of the means (ties by old id).
    bool Compute(const float* params, int count);
    const uint32_t* GetPermutation() const { return perm_; }
    // Reorders the block in place (either layout) by the last permutation and
    // composes `parents` (device, nullable: identity) into GetParents():
    // parents'[i] = parents[perm[i]].
    bool Apply(float* params, int count, bool bf16_sh, const int* parents);
    const int* GetParents() const { return parents_.get(); }
    // out[i] = parents[perm[i]] for another parent map (device, count entries).
    bool Compose(const int* parents, int* out);

private:
    cudaStream_t stream_ = nullptr;
    DeviceArray<uint32_t> keys_[2], ids_[2];
    DeviceArray<uint8_t> sort_scratch_;
    DeviceArray<int> bounds_, parents_;
    DeviceArray<float> block_;
    const uint32_t* perm_ = nullptr;
    int count_ = 0;
};

}  // namespace gs_native
