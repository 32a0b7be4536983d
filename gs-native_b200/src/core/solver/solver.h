// Drop-in gs_native::Solver (reference: src/core/solver/solver.h:11-68).
//
// Iterate() evaluates dL/dimage of 0.8 * L1 + 0.2 * (1 - SSIM), back-propagates
// it through the renderer's last frame to the screen-space Gaussian gradients,
// maps them to the 58 parameters and applies one Adam step (beta 0.9 / 0.999,
// eps 1e-15) in place on the GaussianBuffers. Same arguments, return values and
// buffer semantics as the reference, including the per-step bias-correction
// counter, ResetOpacityHistory() and the parent-id remap of the Adam history
// after density control. Must be paired with gs_native::Renderer of this
// library (it reads the renderer's frame buffers, like the reference does).
//
// Additions: an explicit stream, configurable per-group learning rates (the
// reference hard-codes them, solver.cu:666-681), an optional FP64 loss/PSNR
// reduction, and optional fused accumulation of the density-control
// statistics.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "core/render/renderer.h"
#include "core/types/buffers.h"
#include "util/device_array.h"

namespace gsn {
struct StepFrame;
}

namespace gs_native {

// Learning rates per parameter group; position comes from Iterate().
struct LearningRates {
    float scale = 0.005f;
    float rotation = 0.001f;
    float opacity = 0.025f;
    float sh_dc = 0.0025f;
    float sh_rest = 0.0025f / 20.0f;
};

class Solver {
public:
    Solver() = default;
    ~Solver();

    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    bool Iterate(const CameraParams& camera, const Renderer& renderer, const float* image, const uint8_t* target,
                 GaussianBuffers& gaussians, float position_learning_rate, int sh_degree);

    bool ResetOpacityHistory();

    bool RemapGaussians(const int* parent_ids, int gaussian_count);

    const float* GetProjectionStatistics() const { return stats_.get(); }
    const float* GetAbsoluteProjectionStatistics() const { return abs_stats_.get(); }

    // ---- extensions
    void SetStream(cudaStream_t stream) { stream_ = stream; }
    void SetLearningRates(const LearningRates& lr) { lr_ = lr; }
    const LearningRates& GetLearningRates() const { return lr_; }
    // When enabled, Iterate() also reduces the loss (FP64) into GetLossDevice():
    // [loss, mean L1, mean SSIM, PSNR dB].
    void SetComputeLoss(bool enabled) { compute_loss_ = enabled; }
    const double* GetLossDevice() const { return loss_.get() ? loss_.get() + 3 : nullptr; }
    // Optional fused accumulation of the density statistics (pointers owned by
    // the caller, all three or none); equivalent to calling
    // DensityController::AccumulateStatistics after Iterate().
    // Statistics of the learned density policy, updated with the density
    // accumulators for visible Gaussians (null: off): round maximum of the
    // screen radius, round sums of depth and depth^2, and the step's gradient
    // norms of mean, log-scale, opacity and SH (float4 per Gaussian).
    void SetLearnedStatistics(float* max_radius, float* depth_sum, float* depth_sq, float4* last_grad) {
        ls_max_radius_ = max_radius;
        ls_depth_sum_ = depth_sum;
        ls_depth_sq_ = depth_sq;
        ls_last_grad_ = last_grad;
    }
    void SetDensityAccumulators(float* gradient_sums, float* absolute_sums, unsigned int* counts) {
        acc_grad_ = gradient_sums;
        acc_abs_ = absolute_sums;
        acc_count_ = counts;
    }
    const float* GetImageGradients() const { return image_gradients_.get(); }
    const float* GetScreenGradients() const { return screen_.get(); }
    float* GetFirstMoments() { return m_.get(); }
    float* GetSecondMoments() { return v_.get(); }
    int GetGaussianCapacity() const { return gaussian_count_; }
    uint64_t GetIteration() const { return iteration_; }
    // Batched form: when set, the loss target, the camera of the update, the
    // position learning rate and Adam's bias corrections are read from this
    // device frame (written on the device at the start of each step).
    void SetStepFrame(const gsn::StepFrame* frame) { frame_ = frame; }
    // Precision form: parameters and moments in the 10 fp32 + 48 bf16 row
    // layout (34 float rows of stride N); SH updates use stochastic rounding.
    // Changing the layout drops the Adam history.
    void SetBf16Sh(bool enabled);
    bool GetBf16Sh() const { return bf16_sh_; }
    // The L1+SSIM gradient on the tcgen05 tensor cores (banded-Toeplitz filter
    // GEMMs, hi/lo bf16 split, fp32 accumulation). On by default in the
    // precision form; can be switched independently.
    void SetTensorCoreLoss(bool enabled) { tensor_core_loss_ = enabled; }
    // Visibility-masked (sparse) Adam: Gaussians without a tile in the frame
    // (the renderer's rectangle count is 0) keep their parameters and moments;
    // the reference updates all of them every iteration (solver.cu:912-915).
    void SetSparseAdam(bool enabled) { sparse_adam_ = enabled; }
    bool GetSparseAdam() const { return sparse_adam_; }
    // Lazy moment decay for the sparse update: a Gaussian that skipped k steps has
    // its moments decayed by 0.9^k and 0.999^k before its next update, as k dense
    // steps with a zero gradient would have decayed them (its parameters do not
    // take those steps' momentum moves). Eager steps only: an update through a
    // captured step frame (CUDA graph) is refused.
    void SetLazyMomentDecay(bool enabled) { lazy_moments_ = enabled; }
    bool GetLazyMomentDecay() const { return lazy_moments_; }
    bool GetTensorCoreLoss() const { return tensor_core_loss_; }
    // Device status word of the tensor-core passes: 0, or GSN_ERR_TIMEOUT.
    const int* GetStatusDevice() const { return status_.get(); }
    void SetIteration(uint64_t iteration) { iteration_ = iteration; }

    // Stage entry points (used by Iterate and by the C ABI).
    bool ComputeImageGradients(const CameraParams& camera, const float* image, const uint8_t* target);
    bool ComputeScreenGradients(const CameraParams& camera, const Renderer& renderer, const GaussianBuffers& g,
                                const float* image);
    // Maps the screen-space gradients to parameters; with `adam` false the 58 x N
    // gradients are written to `grads_out` instead of being applied.
    bool UpdateGaussians(const CameraParams& camera, const Renderer& renderer, GaussianBuffers& g,
                         float position_learning_rate, int sh_degree, bool adam, float* grads_out);

private:
    cudaStream_t stream_ = nullptr;
    LearningRates lr_;
    bool compute_loss_ = false;
    DeviceArray<float> image_gradients_;
    int64_t pixel_capacity_ = 0;
    DeviceArray<float> screen_;     // [N][12]
    DeviceArray<float> stats_;      // 2 x N
    DeviceArray<float> abs_stats_;  // 2 x N
    DeviceArray<float> m_, v_;      // 58 x N, stride == gaussian_count_
    DeviceArray<double> loss_;      // [0..2] sums, [3..6] finalised
    int gaussian_count_ = 0;
    size_t per_gaussian_capacity_ = 0;
    uint64_t iteration_ = 0;
    float* acc_grad_ = nullptr;
    float* ls_max_radius_ = nullptr;
    float* ls_depth_sum_ = nullptr;
    float* ls_depth_sq_ = nullptr;
    float4* ls_last_grad_ = nullptr;
    float* acc_abs_ = nullptr;
    unsigned int* acc_count_ = nullptr;
    const gsn::StepFrame* frame_ = nullptr;
    bool bf16_sh_ = false;
    bool tensor_core_loss_ = false;
    bool sparse_adam_ = false;
    bool lazy_moments_ = false;
    DeviceArray<uint32_t> last_step_;  // [N] step of each Gaussian's last update, 0: unknown
    int last_step_count_ = 0;          // Gaussians last_step_ is valid for (0 after a remap)
    bool fast_loss_ = false;  // set by Iterate from the renderer's fast blend setting
    DeviceArray<int> status_;
};

}  // namespace gs_native
