// gs_native::TrainingGraph: capture and replay of the training iteration.
#include "core/graph/training_graph.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "kernels.h"
#include "profile.h"

namespace gs_native {

namespace {

constexpr int kBatchCapacity = 4096;  // schedule entries per upload

}  // namespace

TrainingGraph::~TrainingGraph() { Release(); }

void TrainingGraph::Release() {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (capture_stream_) cudaStreamDestroy(capture_stream_);
    exec_ = nullptr;
    graph_ = nullptr;
    capture_stream_ = nullptr;
    if (renderer_) renderer_->SetDeviceCamera(nullptr);
    if (solver_) solver_->SetStepFrame(nullptr);
    renderer_ = nullptr;
    solver_ = nullptr;
}

bool TrainingGraph::Capture(Renderer& renderer, Solver& solver, GaussianBuffers& gaussians,
                            const std::vector<CameraParams>& cameras, const uint8_t* device_targets,
                            size_t target_stride, const float background[3], float* device_image, int sh_degree,
                            int64_t record_capacity, cudaStream_t stream) {
    Release();
    if (cameras.empty() || !device_targets || !background || !device_image || record_capacity <= 0 ||
        gaussians.gaussian_count_ <= 0 || !gaussians.gaussians_)
        return false;
    const CameraParams& c0 = cameras[0];
    for (const CameraParams& c : cameras)
        if (c.width_ != c0.width_ || c.height_ != c0.height_ || c.tile_count_x_ != c0.tile_count_x_ ||
            c.tile_count_y_ != c0.tile_count_y_)
            return false;
    stream_ = stream;
    view_count_ = static_cast<int>(cameras.size());
    batch_capacity_ = kBatchCapacity;
    if (!cameras_.Reserve(cameras.size()) || !views_.Reserve(batch_capacity_) ||
        !schedule_.Reserve(4 * static_cast<size_t>(batch_capacity_)) || !control_.Reserve(2) ||
        !frame_.Reserve(sizeof(gsn::StepFrame)))
        return false;
    std::vector<gsn_camera> cams(cameras.size());
    for (size_t k = 0; k < cameras.size(); ++k) cams[k] = AsGsnCamera(cameras[k]);
    if (cudaMemcpyAsync(cameras_.get(), cams.data(), cams.size() * sizeof(gsn_camera), cudaMemcpyHostToDevice,
                        stream) != cudaSuccess ||
        cudaMemsetAsync(control_.get(), 0, 2 * sizeof(int), stream) != cudaSuccess ||
        cudaMemsetAsync(views_.get(), 0, batch_capacity_ * sizeof(int), stream) != cudaSuccess ||
        cudaMemsetAsync(schedule_.get(), 0, 4 * batch_capacity_ * sizeof(float), stream) != cudaSuccess)
        return false;

    renderer.SetStream(stream);
    solver.SetStream(stream);
    if (!renderer.SetRecordCapacity(record_capacity)) return false;
    // eager pass without the update: every buffer of the step is reserved
    // before the capture, which must not allocate or synchronise
    if (!renderer.Render(gaussians, c0, background, device_image, sh_degree) ||
        !solver.ComputeImageGradients(c0, device_image, device_targets) ||
        !solver.ComputeScreenGradients(c0, renderer, gaussians, device_image) ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return false;

    auto* frame = reinterpret_cast<gsn::StepFrame*>(frame_.get());
    gsn::StepSchedule s{};
    s.cameras = cameras_.get();
    s.targets = device_targets;
    s.target_stride = static_cast<int64_t>(target_stride);
    s.views = views_.get();
    s.position_lr = schedule_.get();
    s.c1 = schedule_.get() + batch_capacity_;
    s.c2 = schedule_.get() + 2 * batch_capacity_;
    s.seeds = reinterpret_cast<const uint32_t*>(schedule_.get() + 3 * batch_capacity_);
    s.cursor = control_.get();
    s.status = control_.get() + 1;
    s.overflow = renderer.GetOverflowFlag();
    s.steps = batch_capacity_;
    s.view_count = view_count_;

    renderer_ = &renderer;
    solver_ = &solver;
    renderer.SetDeviceCamera(&frame->cam);
    solver.SetStepFrame(frame);
    // the capture runs on a stream of its own (the caller's may be the legacy
    // default stream, which cannot be captured); replays go to the caller's
    if (cudaStreamCreateWithFlags(&capture_stream_, cudaStreamNonBlocking) != cudaSuccess) {
        capture_stream_ = nullptr;
        Release();
        return false;
    }
    renderer.SetStream(capture_stream_);
    solver.SetStream(capture_stream_);
    const bool profiling = gsn::profile_enabled();
    gsn::profile_enable(false);
    const uint64_t iteration = solver.GetIteration();
    const uint64_t launches0 = gsn::launch_count();
    bool ok = cudaStreamBeginCapture(capture_stream_, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        ok = gsn::launch_advance_frame(s, frame, capture_stream_) == GSN_OK &&
             renderer.Render(gaussians, c0, background, device_image, sh_degree) &&
             solver.Iterate(c0, renderer, device_image, device_targets, gaussians, 0.0f, sh_degree);
        cudaGraph_t graph = nullptr;
        const bool ended = cudaStreamEndCapture(capture_stream_, &graph) == cudaSuccess;
        ok = ok && ended && graph;
        graph_ = graph;
    }
    launches_per_step_ = static_cast<int>(gsn::launch_count() - launches0);
    solver.SetIteration(iteration);
    renderer.SetStream(stream);
    solver.SetStream(stream);
    gsn::profile_enable(profiling);
    if (ok) ok = cudaGraphInstantiate(&exec_, graph_, 0) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        Release();
        return false;
    }
    return true;
}

bool TrainingGraph::Run(const int* views, const float* position_lrs, int steps) {
    if (!exec_ || steps < 0 || (steps > 0 && (!views || !position_lrs))) return false;
    for (int done = 0; done < steps;) {
        const int n = std::min(steps - done, batch_capacity_);
        for (int k = 0; k < n; ++k)
            if (views[done + k] < 0 || views[done + k] >= view_count_) return false;
        // c1, c2 exactly as Solver::UpdateGaussians computes them (FP64 on the host)
        host_schedule_.assign(4 * static_cast<size_t>(n), 0.0f);
        const uint64_t t0 = solver_->GetIteration();
        for (int k = 0; k < n; ++k) {
            const double t = static_cast<double>(t0 + k + 1);
            host_schedule_[k] = position_lrs[done + k];
            host_schedule_[n + k] = static_cast<float>(1.0 / (1.0 - std::pow(0.9, t)));
            host_schedule_[2 * n + k] = static_cast<float>(1.0 / (1.0 - std::pow(0.999, t)));
            // the seed is the Adam step number, as in the eager update
            const uint32_t seed = static_cast<uint32_t>(t0 + k + 1);
            std::memcpy(&host_schedule_[3 * n + k], &seed, sizeof(seed));
        }
        float* dev = schedule_.get();
        if (cudaMemcpyAsync(views_.get(), views + done, n * sizeof(int), cudaMemcpyHostToDevice, stream_) !=
                cudaSuccess ||
            cudaMemcpyAsync(dev, host_schedule_.data(), n * sizeof(float), cudaMemcpyHostToDevice, stream_) !=
                cudaSuccess ||
            cudaMemcpyAsync(dev + batch_capacity_, host_schedule_.data() + n, n * sizeof(float),
                            cudaMemcpyHostToDevice, stream_) != cudaSuccess ||
            cudaMemcpyAsync(dev + 2 * batch_capacity_, host_schedule_.data() + 2 * n, n * sizeof(float),
                            cudaMemcpyHostToDevice, stream_) != cudaSuccess ||
            cudaMemcpyAsync(dev + 3 * batch_capacity_, host_schedule_.data() + 3 * n, n * sizeof(float),
                            cudaMemcpyHostToDevice, stream_) != cudaSuccess ||
            cudaMemsetAsync(control_.get(), 0, sizeof(int), stream_) != cudaSuccess)
            return false;
        for (int k = 0; k < n; ++k)
            if (cudaGraphLaunch(exec_, stream_) != cudaSuccess) return false;
        gsn::note_launch(n * launches_per_step_);
        solver_->SetIteration(t0 + n);
        done += n;
    }
    return true;
}

int TrainingGraph::Check() {
    if (!exec_) return GSN_ERR_NOT_READY;
    int status[2] = {0, 0};
    if (cudaMemcpyAsync(&status[0], control_.get() + 1, sizeof(int), cudaMemcpyDeviceToHost, stream_) !=
            cudaSuccess ||
        cudaMemcpyAsync(&status[1], renderer_->GetOverflowFlag(), sizeof(int), cudaMemcpyDeviceToHost, stream_) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
        return GSN_ERR_CUDA;
    if (status[0] != 0 || status[1] != 0) {
        // the status is sticky until reported
        if (cudaMemsetAsync(control_.get() + 1, 0, sizeof(int), stream_) != cudaSuccess) return GSN_ERR_CUDA;
        return GSN_ERR_CAPACITY;
    }
    return GSN_OK;
}

}  // namespace gs_native
