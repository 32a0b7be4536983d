// Batched form of the training iteration: one CUDA graph holds the whole step
// (frame advance -> projection -> depth sort -> record scan -> emit -> tile sort
// -> tile ranges -> forward blend -> L1+SSIM gradient -> backward blend ->
// chain rule + Adam) over max-capacity buffers with device-side counts, and is
// replayed once per iteration. The per-step inputs - view, position learning
// rate and Adam bias corrections - come from a device schedule that a one-warp
// frame kernel reads at the start of each replay, so a run of K iterations is
// K graph launches with no host work or synchronisation in between.
//
// The arithmetic of a step is the eager Renderer::Render + Solver::Iterate's;
// only where the camera, target and step scalars are read from differs. The
// reference has no batched form (it runs each stage from the host and reads
// the record count back every frame, renderer.cu:480-500).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "core/render/renderer.h"
#include "core/solver/solver.h"
#include "core/types/buffers.h"
#include "util/device_array.h"

namespace gsn {
struct StepFrame;
}

namespace gs_native {

class TrainingGraph {
public:
    TrainingGraph() = default;
    ~TrainingGraph();
    TrainingGraph(const TrainingGraph&) = delete;
    TrainingGraph& operator=(const TrainingGraph&) = delete;

    // Captures one iteration over `cameras` (all of the same resolution) whose
    // training targets are resident at device_targets + v * target_stride (u8
    // HWC). The renderer switches to a fixed record capacity (`record_capacity`
    // tile records); a step that would exceed it is reported by Check(). The
    // renderer, solver and Gaussian buffers must stay alive and the Gaussian
    // count and parameter block unchanged while the graph is used.
    bool Capture(Renderer& renderer, Solver& solver, GaussianBuffers& gaussians,
                 const std::vector<CameraParams>& cameras, const uint8_t* device_targets, size_t target_stride,
                 const float background[3], float* device_image, int sh_degree, int64_t record_capacity,
                 cudaStream_t stream);
    // Runs `steps` iterations, view views[k] with position learning rate
    // position_lrs[k]; Adam's step counter continues from the solver's. The
    // launches are asynchronous on the capture stream.
    bool Run(const int* views, const float* position_lrs, int steps);
    // Synchronises and returns GSN_OK, or GSN_ERR_CAPACITY if a step's records
    // exceeded the capacity (that step's image and update are incomplete).
    int Check();
    // Kernel launches of one replayed step.
    int LaunchesPerStep() const { return launches_per_step_; }
    bool Captured() const { return exec_ != nullptr; }
    // Releases the graph and detaches the renderer and solver from the frame.
    void Release();

private:
    Renderer* renderer_ = nullptr;
    Solver* solver_ = nullptr;
    cudaStream_t stream_ = nullptr;          // replays
    cudaStream_t capture_stream_ = nullptr;  // owned; used for the capture only
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    int view_count_ = 0;
    int launches_per_step_ = 0;
    int batch_capacity_ = 0;
    DeviceArray<gsn_camera> cameras_;
    DeviceArray<int> views_;
    DeviceArray<float> schedule_;    // position lr, c1, c2, seed planes of batch_capacity_
    DeviceArray<int> control_;       // [0] cursor, [1] status
    DeviceArray<unsigned char> frame_;
    std::vector<float> host_schedule_;
};

}  // namespace gs_native
