// gs_native::Solver over the sm_100a kernels (reference behaviour:
// src/core/solver/solver.cu:693-929).
#include "core/solver/solver.h"

#include <algorithm>
#include <cmath>

#include "kernels.h"
#include "profile.h"

namespace gs_native {

Solver::~Solver() = default;

namespace {

size_t PhysicalRows(bool bf16_sh) { return bf16_sh ? 34 : kMaxParamCount; }

}  // namespace

void Solver::SetBf16Sh(bool enabled) {
    if (enabled == bf16_sh_) return;
    bf16_sh_ = enabled;
    tensor_core_loss_ = enabled;
    m_.Reset();
    v_.Reset();
    gaussian_count_ = 0;
    iteration_ = 0;
}

bool Solver::Iterate(const CameraParams& camera, const Renderer& renderer, const float* image, const uint8_t* target,
                     GaussianBuffers& gaussians, float position_learning_rate, int sh_degree) {
    // the fast blend forms also take the fast SSIM moments
    fast_loss_ = renderer.GetFastBlend();
    const bool ok = ComputeImageGradients(camera, image, target);
    fast_loss_ = false;
    if (!ok) return false;
    if (!ComputeScreenGradients(camera, renderer, gaussians, image)) return false;
    return UpdateGaussians(camera, renderer, gaussians, position_learning_rate, sh_degree, true, nullptr);
}

bool Solver::ResetOpacityHistory() {
    if (gaussian_count_ == 0) return true;
    const int64_t offset = static_cast<int64_t>(kOpacityIndex) * gaussian_count_;
    const size_t bytes = static_cast<size_t>(gaussian_count_) * sizeof(float);
    return cudaMemsetAsync(m_.get() + offset, 0, bytes, stream_) == cudaSuccess &&
           cudaMemsetAsync(v_.get() + offset, 0, bytes, stream_) == cudaSuccess;
}

bool Solver::RemapGaussians(const int* parent_ids, int gaussian_count) {
    if (gaussian_count < 0) return false;
    last_step_count_ = 0;  // step records restart as unknown after any remap
    if (gaussian_count == 0) {
        m_.Reset();
        v_.Reset();
        gaussian_count_ = 0;
        return true;
    }
    const size_t n = static_cast<size_t>(gaussian_count);
    if (n > per_gaussian_capacity_) {
        if (!screen_.Reserve(n * 12) || !stats_.Reserve(2 * n) || !abs_stats_.Reserve(2 * n)) return false;
        if (cudaMemsetAsync(screen_.get(), 0, n * 12 * sizeof(float), stream_) != cudaSuccess) return false;
        per_gaussian_capacity_ = n;
    }
    DeviceArray<float> m, v;
    if (!m.Reserve(n * PhysicalRows(bf16_sh_)) || !v.Reserve(n * PhysicalRows(bf16_sh_))) return false;
    if (gsn::launch_remap_moments(parent_ids, m_.get(), v_.get(), m.get(), v.get(), m_.get() ? gaussian_count_ : 0,
                                  gaussian_count, bf16_sh_, stream_) != GSN_OK)
        return false;
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return false;
    m_ = std::move(m);
    v_ = std::move(v);
    gaussian_count_ = gaussian_count;
    return true;
}

bool Solver::ComputeImageGradients(const CameraParams& camera, const float* image, const uint8_t* target) {
    if (!image || !target || camera.width_ <= 0 || camera.height_ <= 0) return false;
    const int64_t pixels = static_cast<int64_t>(camera.width_) * camera.height_;
    if (pixels > pixel_capacity_) {
        if (!image_gradients_.Reserve(static_cast<size_t>(pixels) * 3)) return false;
        pixel_capacity_ = pixels;
    }
    double* sums = nullptr;
    if (compute_loss_) {
        if (!loss_.Reserve(8)) return false;
        sums = loss_.get();
    }
    gsn::stage_mark(stream_, gsn::kStageLossGradient);
    if (tensor_core_loss_) {
        if (!status_.get()) {
            if (!status_.Reserve(1) || cudaMemsetAsync(status_.get(), 0, sizeof(int), stream_) != cudaSuccess)
                return false;
        }
        if (gsn::launch_loss_gradient_tc(image, target, frame_, image_gradients_.get(), camera.width_,
                                         camera.height_, sums, status_.get(), stream_) != GSN_OK)
            return false;
    } else if (gsn::launch_loss_gradient(image, target, frame_, image_gradients_.get(), camera.width_,
                                         camera.height_, sums, stream_, fast_loss_) != GSN_OK) {
        return false;
    }
    if (sums && gsn::launch_finalize_loss(sums, camera.width_, camera.height_, loss_.get() + 3, stream_) != GSN_OK)
        return false;
    return true;
}

bool Solver::ComputeScreenGradients(const CameraParams& camera, const Renderer& renderer, const GaussianBuffers& g,
                                    const float* image) {
    const int count = g.gaussian_count_;
    if (count == 0) return true;
    const int64_t pixels = static_cast<int64_t>(camera.width_) * camera.height_;
    const int64_t tiles = static_cast<int64_t>(camera.tile_count_x_) * camera.tile_count_y_;
    if (count < 0 || !g.gaussians_ || !image || !image_gradients_.get() || camera.width_ <= 0 ||
        camera.height_ <= 0 || pixels > pixel_capacity_ || camera.tile_count_x_ <= 0 || camera.tile_count_y_ <= 0 ||
        tiles > renderer.GetTileCapacity() || count > renderer.GetGaussianCapacity() ||
        count != renderer.GetLastGaussianCount() || !renderer.GetTileGaussianOffsets() || !renderer.GetMeans() ||
        !renderer.GetConicOpacities() || !renderer.GetColors())
        return false;
    if (count != gaussian_count_) {
        if (iteration_ != 0 || !RemapGaussians(nullptr, count)) return false;
    }
    gsn::stage_mark(stream_, gsn::kStageRasterBackward);
    if (cudaMemsetAsync(screen_.get(), 0, static_cast<size_t>(count) * 12 * sizeof(float), stream_) != cudaSuccess)
        return false;
    gsn::RasterBackwardArgs a;
    a.tile_ids = reinterpret_cast<const uint32_t*>(renderer.GetTileGaussianIds());
    a.tile_offsets = renderer.GetTileGaussianOffsets();
    a.means = renderer.GetMeans();
    a.conic_opacity = renderer.GetConicOpacities();
    a.colors = renderer.GetColors();
    a.image = image;
    a.image_grad = image_gradients_.get();
    a.contributors = renderer.GetContributors();
    a.record_warps = renderer.GetRecordWarps();
    a.record_words = renderer.GetRecordWords();
    a.fast = renderer.GetFastBlend();
    a.cam = AsGsnCamera(camera);
    a.grad_out = screen_.get();
    return gsn::launch_raster_backward(a, stream_) == GSN_OK;
}

bool Solver::UpdateGaussians(const CameraParams& camera, const Renderer& renderer, GaussianBuffers& g,
                             float position_learning_rate, int sh_degree, bool adam, float* grads_out) {
    const int count = g.gaussian_count_;
    if (count == 0) return true;
    if (count < 0 || count != gaussian_count_ || !g.gaussians_ || !m_.get() || !v_.get() ||
        !std::isfinite(position_learning_rate) || position_learning_rate < 0 || !renderer.GetTileCounts())
        return false;
    const uint64_t iteration = iteration_ + 1;
    gsn::GaussianUpdateArgs a{};
    a.params = g.gaussians_;
    a.m = adam ? m_.get() : nullptr;
    a.v = adam ? v_.get() : nullptr;
    a.screen = screen_.get();
    a.tile_counts = renderer.GetTileCounts();
    a.cam = AsGsnCamera(camera);
    a.n = count;
    a.lr[0] = position_learning_rate;
    a.lr[1] = lr_.scale;
    a.lr[2] = lr_.rotation;
    a.lr[3] = lr_.opacity;
    a.lr[4] = lr_.sh_dc;
    a.lr[5] = lr_.sh_rest;
    a.c1 = static_cast<float>(1.0 / (1.0 - std::pow(0.9, static_cast<double>(iteration))));
    a.c2 = static_cast<float>(1.0 / (1.0 - std::pow(0.999, static_cast<double>(iteration))));
    a.stats = stats_.get();
    a.abs_stats = abs_stats_.get();
    if (adam && acc_grad_ && acc_abs_ && acc_count_) {
        a.grad_sums = acc_grad_;
        a.abs_sums = acc_abs_;
        a.obs_counts = acc_count_;
        if (ls_max_radius_ && ls_depth_sum_ && ls_depth_sq_ && ls_last_grad_ && renderer.GetRadii() &&
            renderer.GetDepths()) {
            a.radii = renderer.GetRadii();
            a.depths = renderer.GetDepths();
            a.max_radius = ls_max_radius_;
            a.depth_sum = ls_depth_sum_;
            a.depth_sq = ls_depth_sq_;
            a.last_grad = ls_last_grad_;
        }
    }
    a.grads_out = grads_out;
    a.frame = frame_;
    a.bf16_sh = bf16_sh_;
    a.sparse = sparse_adam_;
    a.seed = static_cast<uint32_t>(iteration);
    if (adam && lazy_moments_) {
        if (!sparse_adam_ || frame_) return false;  // sparse eager updates only
        if (last_step_count_ != count) {
            if (!last_step_.Reserve(static_cast<size_t>(count)) ||
                cudaMemsetAsync(last_step_.get(), 0, static_cast<size_t>(count) * sizeof(uint32_t), stream_) !=
                    cudaSuccess)
                return false;
            last_step_count_ = count;
        }
        a.last_step = last_step_.get();
        a.step = static_cast<uint32_t>(iteration);
    }
    gsn::stage_mark(stream_, gsn::kStageGaussianUpdate);
    if (gsn::launch_gaussian_update(a, std::clamp(sh_degree, 0, 3), stream_) != GSN_OK) return false;
    gsn::stage_mark(stream_, gsn::kStageOther);
    if (adam) iteration_ = iteration;
    return true;
}

}  // namespace gs_native
