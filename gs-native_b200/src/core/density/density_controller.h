// Drop-in gs_native::DensityController (reference:
// src/core/density/density_controller.h:9-83).
//
// Same interface and semantics: per-round statistics, the clone/split/prune
// decision with absolute-gradient splits and optional pruning of large
// Gaussians, Philox-sampled split children, opacity reset, and the ownership
// ping-pong of the parameter block: on success ControlDensity() hands the caller
// a new 58 x N' block it owns and keeps the caller's old block as its spare
// (all Gaussians pruned: the caller receives nullptr / 0). GetHistoryParentIds()
// maps every new Gaussian to the old index whose Adam history it keeps (-1 for
// new ones), GetParentIds() to its source Gaussian.
//
// Additions: an explicit stream, an optional cap on the Gaussian count
// (SetMaxGaussians) and the per-output new-Gaussian flags.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "core/types/buffers.h"
#include "density.h"
#include "util/device_array.h"

namespace gs_native {

class DensityController {
public:
    DensityController() = default;
    ~DensityController();
    DensityController(const DensityController&) = delete;
    DensityController& operator=(const DensityController&) = delete;

    bool Initialize(int gaussian_count, int capacity);

    bool AccumulateStatistics(const float* gradients, const float* radii, const int* gaussian_ids,
                              int observation_count);

    bool AccumulateStatistics(const float* statistics, const float* absolute_statistics, int gaussian_count);

    bool ResetOpacity(float* parameters, int stride, float max_opacity = 0.01f);

    bool ControlDensity(GaussianBuffers& gaussians, float scene_extent, float gradient_threshold = 0.0002f,
                        float percent_dense = 0.01f, float min_opacity = 0.005f, float max_screen_size = 0.0f,
                        unsigned long long seed = 0, int* changes = nullptr, float absolute_gradient_threshold = 0.0f);

    const int* GetHistoryParentIds() const { return history_parent_ids_; }
    const int* GetGaussianCount() const { return control_.get(); }
    const int* GetStatus() const { return control_.get() ? control_.get() + 2 : nullptr; }
    const int* GetParentIds() const { return parent_ids_.get(); }

    // ---- extensions
    void SetStream(cudaStream_t stream) { stream_ = stream; }
    // 0 = unlimited (reference behaviour).
    void SetMaxGaussians(int max_gaussians) { max_gaussians_ = max_gaussians < 0 ? 0 : max_gaussians; }
    // Precision form: parameter blocks in the 10 fp32 + 48 bf16 row layout
    // (34 float rows of stride N); set before the first ControlDensity.
    void SetBf16Sh(bool enabled) { bf16_sh_ = enabled; }
    // Learned proposals for the next ControlDensity: per Gaussian 0 keep,
    // 1 clone, 2 split, 3 prune, or < 0 for the plain threshold rule (device,
    // count entries; nullptr = plain rule for all).
    void SetActionOverride(const int8_t* actions) { actions_ = actions; }
    // Decision codes (0 keep, 1 clone, 2 split, 3 prune) of the last
    // ControlDensity into a device int8 array of the pre-control count.
    bool GetDecisionCodes(int8_t* codes, int count) const;
    // The 16 statistics of the learned policy for the current Gaussians
    // (device [count][16]) from the round statistics and the policy's own
    // per-Gaussian statistics (ls).
    bool ComputeFeatures(const GaussianBuffers& gaussians, float scene_extent, float gradient_threshold,
                         float percent_dense, const gsn::LearnedStatsView& ls, float* features) const;
    const float* GetNewFlags() const { return new_flags_.get(); }
    float* GetGradientSums() { return gradient_sums_.get(); }
    float* GetAbsoluteGradientSums() { return absolute_gradient_sums_.get(); }
    unsigned int* GetObservationCounts() { return observation_counts_.get(); }
    int GetCapacity() const { return capacity_; }
    const float* GetSamples() const { return samples_.get(); }

private:
    bool Reserve(int capacity);

    cudaStream_t stream_ = nullptr;
    float* spare_gaussian_parameters_ = nullptr;
    int* history_parent_ids_ = nullptr;
    int spare_gaussian_stride_ = 0;

    DeviceArray<float> gradient_sums_;
    DeviceArray<float> absolute_gradient_sums_;
    DeviceArray<unsigned int> observation_counts_;
    DeviceArray<float> samples_;
    DeviceArray<int> parent_ids_;
    DeviceArray<float> new_flags_;
    DeviceArray<int4> density_counts_;
    DeviceArray<int4> density_offsets_;
    DeviceArray<int> additions_;
    DeviceArray<int> control_;
    DeviceArray<unsigned char> scan_storage_;
    DeviceArray<unsigned char> int_scan_storage_;
    int* host_control_ = nullptr;  // pinned int[8]
    int capacity_ = 0;
    int parameter_stride_ = 0;
    int random_blocks_ = 0;
    int max_gaussians_ = 0;
    bool bf16_sh_ = false;
    const int8_t* actions_ = nullptr;
    unsigned long long seed_ = 0;
};

}  // namespace gs_native
