// Drop-in trainer gs_native::GaussianSplatting (reference:
// src/core/gaussian_splatting.h:14-53, gaussian_splatting.cpp:23-342), without
// OpenCV: the scene is given as camera parameters, host u8 HWC images and a
// host point cloud instead of cv::Mat / Camera objects.
//
// Same schedule as the reference (all values configurable through
// TrainingOptions, defaults equal to the reference's constants): one training
// camera per iteration in a std::mt19937(0) shuffled order that is re-drawn when
// exhausted (the generator is re-created at every Train call, as in the
// reference); SH degree min(3, it / 1000); position learning rate
// extent * exp(lerp(log 1.6e-4, log 1.6e-6, it / 30000)); statistics accumulated
// while it < 15000; density control every 100 iterations after 500 with
// prune-large after 3000; opacity capped at 0.8 every 500 and 0.01 every 3000
// iterations. Training images stay resident in device memory; the reference
// uploads one per iteration from pageable host memory.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "core/density/density_controller.h"
#include "core/density/density_mlp.h"
#include "core/graph/training_graph.h"
#include "core/render/renderer.h"
#include "core/solver/solver.h"
#include "core/spatial/spatial_order.h"
#include "core/types/buffers.h"
#include "util/device_array.h"

namespace gs_native {

struct TrainingScene {
    std::vector<CameraParams> train_cameras;
    std::vector<const uint8_t*> train_images;  // host HWC u8 (width * height * 3 bytes), not owned
    const float* point_positions = nullptr;     // host xyz, point_count entries
    const float* point_colors = nullptr;        // host rgb in [0, 1]
    int point_count = 0;
};

struct TrainingOptions {
    int sh_degree_interval = 1000;
    int max_sh_degree = 3;
    float position_lr_init = 0.00016f;
    float position_lr_final = 0.0000016f;
    int position_lr_steps = 30000;
    LearningRates lr;  // non-position groups (solver.cu:666-681)
    int densify_from = 500;       // density control when it > densify_from ...
    int densify_until = 15000;    // ... and it < densify_until (statistics too)
    int densify_interval = 100;
    float gradient_threshold = 0.0002f;
    float absolute_gradient_threshold = 0.0008f;
    float percent_dense = 0.01f;
    float min_opacity = 0.005f;
    int prune_large_after = 3000;
    int opacity_cap_interval = 500;
    float opacity_cap = 0.8f;
    int opacity_reset_interval = 3000;
    float opacity_reset = 0.01f;
    float background[3] = {0.0f, 0.0f, 0.0f};
    int max_gaussians = 0;  // 0 = unlimited (reference behaviour)
    unsigned long long density_seed = 0;
    float initial_opacity = 0.1f;  // initial opacity logit log(o / (1 - o))
    // gs-native extensions
    bool bf16_sh = false;  // precision form: SH rows and their moments in bf16 (34-row block)
    bool graph = false;    // steady-state iterations (after densify_until) as CUDA-graph replays
    // learned density policy: the MLP's proposals (SetDensityMlp) replace the
    // threshold rule where its softmax confidence reaches learned_confidence
    bool learned_density = false;
    float learned_confidence = 0.9f;
    bool log_density = false;  // keep the statistics and decisions of the last control step (GetDensityLog)
    bool exact_culling = false;  // training renderer emits only records that can contribute (Renderer::SetExactCulling)
    // visibility-masked Adam (Solver::SetSparseAdam): Gaussians outside the view keep p, m, v
    bool sparse_adam = false;
    // Morton order of the Gaussians after initialisation and every density step
    // (SpatialOrder): no value changes, the sparse update skips whole sectors
    bool spatial_order = false;
    bool fast_blend = false;  // training renderer's fast blend arithmetic (Renderer::SetFastBlend)
    bool fp32_ssim = false;   // precision form keeps the fp32 CUDA-core SSIM gradient (not the tcgen05 one)
};

// Statistics, decisions and parent map of the last density-control step
// (device pointers, valid until the next step).
struct DensityLog {
    const float* features = nullptr;  // [before][16] statistics before the decision
    const int8_t* decisions = nullptr;  // [before] 0 keep, 1 clone, 2 split, 3 prune
    const int* parents = nullptr;     // [after] source index of every output Gaussian
    int before = 0, after = 0;
    int steps = 0;                    // control steps logged so far
    int iteration = 0;                // iteration of the last step
};

class GaussianSplatting {
public:
    GaussianSplatting() = default;
    ~GaussianSplatting();

    GaussianSplatting(const GaussianSplatting&) = delete;
    GaussianSplatting& operator=(const GaussianSplatting&) = delete;

    bool Initialize(const TrainingScene& scene, const TrainingOptions& options = TrainingOptions());
    bool Train(int iterations);
    // Renders into a device fp32 HWC image of camera.width_ * camera.height_ * 3.
    bool Render(const CameraParams& camera, float* device_image);
    bool Save(const std::string& path);
    // Replaces the model by a PLY file (Adam history and statistics reset).
    bool Load(const std::string& path);
    // Mean PSNR (dB) of the current model over the given views (host u8 HWC
    // images) and the mean training loss; see EvaluateMetrics.
    bool Evaluate(const std::vector<CameraParams>& cameras, const std::vector<const uint8_t*>& images, double* psnr,
                  double* loss = nullptr);
    // Held-out-view metrics averaged over the views, in FP64 on the GPU: PSNR
    // (dB) of the RGB MSE, SSIM (11x11 Gaussian window, sigma 1.5) and L1, all of
    // the render clamped to [0, 1], plus the training loss of the unclamped
    // render. Any output may be null.
    bool EvaluateMetrics(const std::vector<CameraParams>& cameras, const std::vector<const uint8_t*>& images,
                         double* psnr, double* ssim, double* l1, double* loss);

    void SetStream(cudaStream_t stream);
    const GaussianBuffers& GetGaussians() const { return gaussians_; }
    int GetCompleted() const { return completed_; }
    int GetShDegree() const { return sh_degree_; }
    float GetSceneExtent() const { return scene_extent_; }
    Renderer& GetRenderer() { return renderer_; }
    Solver& GetSolver() { return solver_; }
    DensityController& GetDensity() { return density_; }
    const TrainingOptions& GetOptions() const { return options_; }
    // Resumable checkpoint: parameters in their stored layout, Adam moments and
    // step, the round's density statistics, iteration, camera order and cursor
    // (the reference has none). Load requires Initialize() with the same scene
    // first (the targets are not stored) and the same layout option.
    bool SaveCheckpoint(const std::string& path);
    bool LoadCheckpoint(const std::string& path);
    // Weights of the learned density policy (DensityMlp::kParams floats, host).
    bool SetDensityMlp(const float* weights);
    const DensityLog& GetDensityLog() const { return density_log_; }

private:
    bool InitializeGaussians(const float* positions, const float* colors, int count);
    // Uploads a host 58 x count fp32 block in the active layout (bf16 SH rows
    // for the precision form) and resets the optimiser and density state.
    bool SetParameters(const float* host_params, int count);
    // The parameters as a host 58 x count fp32 block (bf16 SH rows widened).
    bool GetParameters(std::vector<float>& out) const;
    size_t PhysicalRows() const;
    bool ControlDensity();
    bool Step();
    void NextCamera();
    // Runs `iterations` steady-state steps as graph replays (after densify_until).
    bool GraphSteps(int iterations);
    float PositionLearningRate(int iteration) const;

    cudaStream_t stream_ = nullptr;
    TrainingOptions options_;
    std::vector<CameraParams> cameras_;
    DeviceArray<uint8_t> targets_;
    size_t target_stride_ = 0;  // bytes per resident training image
    GaussianBuffers gaussians_;
    Renderer renderer_;
    SpatialOrder spatial_;
    DeviceArray<int> log_parents_;  // density-log parent map composed with the spatial order
    Renderer eval_renderer_;  // Render / Evaluate (the training renderer may be bound to a graph)
    Solver solver_;
    DensityController density_;
    DeviceArray<float> image_;
    size_t image_capacity_ = 0;
    std::vector<int> camera_order_;
    int camera_cursor_ = 0;
    int completed_ = 0;
    int sh_degree_ = 0;
    float scene_extent_ = 0.0f;
    TrainingGraph graph_;
    std::mt19937 generator_;
    float scene_centre_[3] = {0.0f, 0.0f, 0.0f};
    DensityMlp mlp_;
    bool mlp_ready_ = false;
    // statistics of the learned policy beyond the round statistics (see
    // LearnedStatsView): round max radius, depth sums, last-step gradient
    // norms, and each Gaussian's birth iteration
    bool ResetLearnedStatistics(int count, const int* history_parents, int prev_count);
    DeviceArray<float> ls_max_radius_, ls_depth_sum_, ls_depth_sq_;
    DeviceArray<float4> ls_last_grad_;
    DeviceArray<int> ls_birth_, ls_birth_next_;
    int ls_count_ = 0;
    DeviceArray<float> density_features_;
    DeviceArray<int8_t> density_actions_;
    DeviceArray<int8_t> density_codes_;
    DensityLog density_log_;
};

}  // namespace gs_native
