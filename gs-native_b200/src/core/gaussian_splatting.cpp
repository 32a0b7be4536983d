// gs_native::GaussianSplatting trainer (reference behaviour:
// src/core/gaussian_splatting.cpp:23-342).
#include "core/gaussian_splatting.h"

#include <algorithm>
#include <array>
#include <climits>
#include <cstring>
#include <cmath>
#include <limits>
#include <numeric>
#include <fstream>
#include <random>

#include "core/knn/knn.h"
#include "io/ply.h"
#include "kernels.h"

namespace gs_native {

GaussianSplatting::~GaussianSplatting() {
    graph_.Release();
    cudaFree(gaussians_.gaussians_);
}

void GaussianSplatting::SetStream(cudaStream_t stream) {
    stream_ = stream;
    graph_.Release();
    renderer_.SetStream(stream);
    solver_.SetStream(stream);
    density_.SetStream(stream);
}

bool GaussianSplatting::Initialize(const TrainingScene& scene, const TrainingOptions& options) {
    if (gaussians_.gaussians_ || scene.train_cameras.empty() || scene.train_cameras.size() != scene.train_images.size() ||
        scene.point_count <= 0 || !scene.point_positions || !scene.point_colors)
        return false;
    size_t pixels = 0;
    for (size_t i = 0; i < scene.train_cameras.size(); ++i) {
        const CameraParams& c = scene.train_cameras[i];
        if (!scene.train_images[i] || c.width_ <= 0 || c.height_ <= 0 || c.tile_count_x_ != (c.width_ + 15) / 16 ||
            c.tile_count_y_ != (c.height_ + 15) / 16)
            return false;
        pixels = std::max(pixels, static_cast<size_t>(c.width_) * c.height_);
    }
    options_ = options;
    cameras_ = scene.train_cameras;
    // scene extent: 1.1 x the largest camera-centre distance from the mean centre
    // (gaussian_splatting.cpp:46-71)
    double mean[3] = {0, 0, 0};
    std::vector<std::array<double, 3>> centers(cameras_.size());
    for (size_t k = 0; k < cameras_.size(); ++k) {
        for (int a = 0; a < 3; ++a) {
            double c = 0;
            for (int r = 0; r < 3; ++r) c -= double(cameras_[k].R_c_w_[r * 3 + a]) * cameras_[k].t_c_w_[r];
            centers[k][a] = c;
            mean[a] += c / cameras_.size();
        }
    }
    double extent = 0;
    for (const auto& c : centers)
        extent = std::max(extent, std::sqrt((c[0] - mean[0]) * (c[0] - mean[0]) + (c[1] - mean[1]) * (c[1] - mean[1]) +
                                            (c[2] - mean[2]) * (c[2] - mean[2])));
    scene_extent_ = static_cast<float>(extent) * 1.1f;
    for (int a = 0; a < 3; ++a) scene_centre_[a] = static_cast<float>(mean[a]);
    if (scene_extent_ == 0.0f) {
        for (int i = 0; i < scene.point_count; ++i) {
            const float* p = scene.point_positions + 3 * i;
            double d = std::sqrt((p[0] - mean[0]) * (p[0] - mean[0]) + (p[1] - mean[1]) * (p[1] - mean[1]) +
                                 (p[2] - mean[2]) * (p[2] - mean[2]));
            scene_extent_ = std::max(scene_extent_, static_cast<float>(d));
        }
        scene_extent_ = std::max(scene_extent_, 1e-6f);
    }
    // resident training targets
    target_stride_ = pixels * 3;
    if (!targets_.Reserve(target_stride_ * cameras_.size()) || !image_.Reserve(pixels * 3)) return false;
    image_capacity_ = pixels * 3;
    for (size_t k = 0; k < cameras_.size(); ++k) {
        const size_t bytes = static_cast<size_t>(cameras_[k].width_) * cameras_[k].height_ * 3;
        if (cudaMemcpyAsync(targets_.get() + k * target_stride_, scene.train_images[k], bytes, cudaMemcpyHostToDevice,
                            stream_) != cudaSuccess)
            return false;
    }
    camera_order_.resize(cameras_.size());
    std::iota(camera_order_.begin(), camera_order_.end(), 0);
    camera_cursor_ = static_cast<int>(camera_order_.size());
    completed_ = 0;
    sh_degree_ = 0;
    solver_.SetLearningRates(options_.lr);
    density_.SetMaxGaussians(options_.max_gaussians);
    renderer_.SetBf16Sh(options_.bf16_sh);
    renderer_.SetExactCulling(options_.exact_culling);
    renderer_.SetFastBlend(options_.fast_blend);
    eval_renderer_.SetBf16Sh(options_.bf16_sh);
    solver_.SetBf16Sh(options_.bf16_sh);
    if (options_.bf16_sh && options_.fp32_ssim) solver_.SetTensorCoreLoss(false);
    density_.SetBf16Sh(options_.bf16_sh);
    solver_.SetSparseAdam(options_.sparse_adam);
    spatial_.SetStream(stream_);
    graph_.Release();
    if (!InitializeGaussians(scene.point_positions, scene.point_colors, scene.point_count)) return false;
    if (options_.spatial_order && gaussians_.gaussian_count_ > 0 &&
        (!spatial_.Compute(gaussians_.gaussians_, gaussians_.gaussian_count_) ||
         !spatial_.Apply(gaussians_.gaussians_, gaussians_.gaussian_count_, options_.bf16_sh, nullptr)))
        return false;
    return cudaStreamSynchronize(stream_) == cudaSuccess;
}

bool GaussianSplatting::InitializeGaussians(const float* positions, const float* colors, int count) {
    std::vector<float> dist(static_cast<size_t>(count), 0.0f);
    if (count >= 2 && !ComputeMeanDist2(positions, count, dist.data(), nullptr, stream_)) return false;
    const size_t N = static_cast<size_t>(count);
    std::vector<float> p(N * kMaxParamCount, 0.0f);
    const float logit = std::log(options_.initial_opacity / (1.0f - options_.initial_opacity));
    for (size_t i = 0; i < N; ++i) {
        const float scale = 0.5f * std::log(std::max(dist[i], 1e-7f));
        for (int a = 0; a < 3; ++a) {
            p[a * N + i] = positions[3 * i + a];
            p[(kLogScaleIndex + a) * N + i] = scale;
            p[(kShIndex + a * 16) * N + i] = (colors[3 * i + a] - 0.5f) / 0.28209479177387814f;
        }
        p[kOpacityIndex * N + i] = logit;
    }
    return SetParameters(p.data(), count);
}

namespace {

// bf16 bits of x, round to nearest even (host side of the precision layout).
uint16_t ToBf16(float x) {
    uint32_t u;
    std::memcpy(&u, &x, sizeof(u));
    if ((u & 0x7f800000u) == 0x7f800000u) return static_cast<uint16_t>(u >> 16 | ((u & 0xffffu) ? 0x40u : 0u));
    u += 0x7fffu + ((u >> 16) & 1u);
    return static_cast<uint16_t>(u >> 16);
}

float FromBf16(uint16_t b) {
    uint32_t u = static_cast<uint32_t>(b) << 16;
    float x;
    std::memcpy(&x, &u, sizeof(x));
    return x;
}

// The precision layout: 10 fp32 rows, then the 48 SH coefficients as 24 rows
// of bf16 pairs (coefficient 2r in the low half of the 32-bit word r * N + i of
// the SH block, 2r + 1 in its high half).
constexpr size_t kGeometryRows = kShIndex;
size_t ShPairIndex(size_t k, size_t N, size_t i) { return ((k >> 1) * N + i) * 2 + (k & 1); }

}  // namespace

size_t GaussianSplatting::PhysicalRows() const { return options_.bf16_sh ? kGeometryRows + 24 : kMaxParamCount; }

bool GaussianSplatting::SetParameters(const float* host_params, int count) {
    const size_t N = static_cast<size_t>(count);
    std::vector<float> block(PhysicalRows() * N);
    if (options_.bf16_sh) {
        std::memcpy(block.data(), host_params, kGeometryRows * N * sizeof(float));
        auto* sh = reinterpret_cast<uint16_t*>(block.data() + kGeometryRows * N);
        for (size_t k = 0; k < kMaxParamCount - kGeometryRows; ++k)
            for (size_t i = 0; i < N; ++i) sh[ShPairIndex(k, N, i)] = ToBf16(host_params[(kGeometryRows + k) * N + i]);
    } else {
        std::memcpy(block.data(), host_params, block.size() * sizeof(float));
    }
    void* dev = nullptr;
    if (DeviceAlloc(&dev, block.size() * sizeof(float)) != cudaSuccess) return false;
    if (cudaMemcpy(dev, block.data(), block.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        !density_.Initialize(count, count) || !solver_.RemapGaussians(nullptr, count)) {
        cudaFree(dev);
        return false;
    }
    graph_.Release();
    cudaFree(gaussians_.gaussians_);
    gaussians_.gaussians_ = static_cast<float*>(dev);
    gaussians_.gaussian_count_ = count;
    return ResetLearnedStatistics(count, nullptr, 0);
}

bool GaussianSplatting::ResetLearnedStatistics(int count, const int* history_parents, int prev_count) {
    const size_t n = static_cast<size_t>(std::max(count, 1));
    // ls_birth_ still holds the previous births (read by the remap): only the
    // destination grows here (Reserve does not keep contents)
    if (!ls_max_radius_.Reserve(n) || !ls_depth_sum_.Reserve(n) || !ls_depth_sq_.Reserve(n) ||
        !ls_last_grad_.Reserve(n) || !ls_birth_next_.Reserve(n))
        return false;
    if (gsn::launch_birth_remap(history_parents, prev_count > 0 ? ls_birth_.get() : nullptr,
                                std::min(prev_count, ls_count_), ls_birth_next_.get(), count, completed_,
                                stream_) != GSN_OK)
        return false;
    std::swap(ls_birth_, ls_birth_next_);
    ls_count_ = count;
    return cudaMemsetAsync(ls_max_radius_.get(), 0, n * sizeof(float), stream_) == cudaSuccess &&
           cudaMemsetAsync(ls_depth_sum_.get(), 0, n * sizeof(float), stream_) == cudaSuccess &&
           cudaMemsetAsync(ls_depth_sq_.get(), 0, n * sizeof(float), stream_) == cudaSuccess &&
           cudaMemsetAsync(ls_last_grad_.get(), 0, n * sizeof(float4), stream_) == cudaSuccess;
}

bool GaussianSplatting::GetParameters(std::vector<float>& out) const {
    const size_t N = static_cast<size_t>(gaussians_.gaussian_count_);
    std::vector<float> block(PhysicalRows() * N);
    if (cudaMemcpy(block.data(), gaussians_.gaussians_, block.size() * sizeof(float), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return false;
    if (!options_.bf16_sh) {
        out = std::move(block);
        return true;
    }
    out.assign(kMaxParamCount * N, 0.0f);
    std::memcpy(out.data(), block.data(), kGeometryRows * N * sizeof(float));
    const auto* sh = reinterpret_cast<const uint16_t*>(block.data() + kGeometryRows * N);
    for (size_t k = 0; k < kMaxParamCount - kGeometryRows; ++k)
        for (size_t i = 0; i < N; ++i) out[(kGeometryRows + k) * N + i] = FromBf16(sh[ShPairIndex(k, N, i)]);
    return true;
}

bool GaussianSplatting::Train(int iterations) {
    if (iterations < 0 || !gaussians_.gaussians_ || cameras_.empty()) return false;
    generator_.seed(0);
    for (int it = 0; it < iterations; ++it) {
        if (gaussians_.gaussian_count_ == 0) return false;
        const int next = completed_ + 1;
        if (options_.graph && completed_ >= options_.densify_until &&
            std::min(options_.max_sh_degree, next / options_.sh_degree_interval) == options_.max_sh_degree &&
            next / options_.sh_degree_interval >= options_.max_sh_degree) {
            if (!GraphSteps(iterations - it)) return false;
            break;
        }
        NextCamera();
        if (!Step()) return false;
    }
    return cudaStreamSynchronize(stream_) == cudaSuccess;
}

void GaussianSplatting::NextCamera() {
    if (camera_cursor_ >= static_cast<int>(camera_order_.size())) {
        std::shuffle(camera_order_.begin(), camera_order_.end(), generator_);
        camera_cursor_ = 0;
    }
}

float GaussianSplatting::PositionLearningRate(int next) const {
    const float fraction = std::min(1.0f, static_cast<float>(next) / static_cast<float>(options_.position_lr_steps));
    return scene_extent_ * std::exp(std::log(options_.position_lr_init) * (1.0f - fraction) +
                                    std::log(options_.position_lr_final) * fraction);
}

bool GaussianSplatting::GraphSteps(int iterations) {
    sh_degree_ = options_.max_sh_degree;
    if (!graph_.Captured()) {
        // twice the largest record buffer the eager steps needed
        const int64_t capacity = std::min<int64_t>(std::max<int64_t>(renderer_.GetRecordCapacity(), 1 << 20) * 2,
                                                   INT_MAX / 2);
        solver_.SetDensityAccumulators(nullptr, nullptr, nullptr);
        solver_.SetLearnedStatistics(nullptr, nullptr, nullptr, nullptr);
        if (!graph_.Capture(renderer_, solver_, gaussians_, cameras_, targets_.get(), target_stride_,
                            options_.background, image_.get(), sh_degree_, capacity, stream_))
            return false;
    }
    std::vector<int> views;
    std::vector<float> lrs;
    for (int done = 0; done < iterations;) {
        const int n = std::min(iterations - done, 4096);
        views.resize(n);
        lrs.resize(n);
        for (int k = 0; k < n; ++k) {
            NextCamera();
            views[k] = camera_order_[camera_cursor_++];
            lrs[k] = PositionLearningRate(completed_ + k + 1);
        }
        if (!graph_.Run(views.data(), lrs.data(), n)) return false;
        completed_ += n;
        done += n;
    }
    return graph_.Check() == GSN_OK;
}

bool GaussianSplatting::Step() {
    const int index = camera_order_[camera_cursor_];
    const CameraParams& camera = cameras_[index];
    const int next = completed_ + 1;
    sh_degree_ = std::min(options_.max_sh_degree, next / options_.sh_degree_interval);
    const float lr = PositionLearningRate(next);
    const uint8_t* target = targets_.get() + static_cast<size_t>(index) * target_stride_;
    if (!renderer_.Render(gaussians_, camera, options_.background, image_.get(), sh_degree_)) return false;
    const bool accumulate = next < options_.densify_until;
    if (accumulate)
        solver_.SetDensityAccumulators(density_.GetGradientSums(), density_.GetAbsoluteGradientSums(),
                                       density_.GetObservationCounts());
    else
        solver_.SetDensityAccumulators(nullptr, nullptr, nullptr);
    if (accumulate && (options_.learned_density || options_.log_density))
        solver_.SetLearnedStatistics(ls_max_radius_.get(), ls_depth_sum_.get(), ls_depth_sq_.get(),
                                     ls_last_grad_.get());
    else
        solver_.SetLearnedStatistics(nullptr, nullptr, nullptr, nullptr);
    if (!solver_.Iterate(camera, renderer_, image_.get(), target, gaussians_, lr, sh_degree_)) return false;
    completed_ = next;
    ++camera_cursor_;
    if (completed_ < options_.densify_until) {
        if (completed_ > options_.densify_from && completed_ % options_.densify_interval == 0 && !ControlDensity())
            return false;
        if (completed_ % options_.opacity_cap_interval == 0) {
            const float cap =
                completed_ % options_.opacity_reset_interval == 0 ? options_.opacity_reset : options_.opacity_cap;
            if (!density_.ResetOpacity(gaussians_.gaussians_, gaussians_.gaussian_count_, cap) ||
                !solver_.ResetOpacityHistory())
                return false;
        }
    }
    return true;
}

bool GaussianSplatting::ControlDensity() {
    int changes[2] = {};
    const float max_screen = completed_ > options_.prune_large_after ? 20.0f : 0.0f;
    const int before = gaussians_.gaussian_count_;
    const bool learned = options_.learned_density && mlp_ready_;
    if (learned || options_.log_density) {
        const gsn::LearnedStatsView ls{ls_max_radius_.get(), ls_depth_sum_.get(), ls_depth_sq_.get(),
                                       ls_last_grad_.get(), ls_birth_.get(), completed_};
        if (!density_features_.Reserve(static_cast<size_t>(std::max(before, 1)) * 16) ||
            !density_.ComputeFeatures(gaussians_, scene_extent_, options_.gradient_threshold,
                                      options_.percent_dense, ls, density_features_.get()))
            return false;
    }
    if (learned) {
        mlp_.SetStream(stream_);
        if (!density_actions_.Reserve(static_cast<size_t>(std::max(before, 1))) ||
            !mlp_.Infer(density_features_.get(), before, options_.learned_confidence, density_actions_.get()))
            return false;
        density_.SetActionOverride(density_actions_.get());
    }
    const bool ok = density_.ControlDensity(gaussians_, scene_extent_, options_.gradient_threshold,
                                            options_.percent_dense, options_.min_opacity, max_screen,
                                            options_.density_seed, changes, options_.absolute_gradient_threshold);
    density_.SetActionOverride(nullptr);
    if (!ok) return false;
    if (options_.log_density) {
        if (!density_codes_.Reserve(static_cast<size_t>(std::max(before, 1))) ||
            !density_.GetDecisionCodes(density_codes_.get(), before))
            return false;
        density_log_.features = density_features_.get();
        density_log_.decisions = density_codes_.get();
        density_log_.parents = density_.GetParentIds();  // composed with the spatial order below
        density_log_.before = before;
        density_log_.after = gaussians_.gaussian_count_;
        density_log_.iteration = completed_;
        ++density_log_.steps;
    }
    const int* history = density_.GetHistoryParentIds();
    const int after = gaussians_.gaussian_count_;
    if (options_.spatial_order && after > 0) {
        // the density step's statistics are zero again, so only the parameters,
        // the Adam history map and the logged parent map follow the permutation
        if (!spatial_.Compute(gaussians_.gaussians_, after) ||
            !spatial_.Apply(gaussians_.gaussians_, after, options_.bf16_sh, history))
            return false;
        if (options_.log_density) {
            if (!log_parents_.Reserve(static_cast<size_t>(after)) ||
                !spatial_.Compose(density_log_.parents, log_parents_.get()))
                return false;
            density_log_.parents = log_parents_.get();
        }
        history = spatial_.GetParents();
    }
    return ResetLearnedStatistics(after, history, before) && solver_.RemapGaussians(history, after);
}

bool GaussianSplatting::SetDensityMlp(const float* weights) {
    mlp_.SetStream(stream_);
    mlp_ready_ = weights && mlp_.SetWeights(weights);
    return mlp_ready_;
}

bool GaussianSplatting::Render(const CameraParams& camera, float* device_image) {
    if (!gaussians_.gaussians_ || !device_image) return false;
    // a renderer of its own: the training renderer's buffers may be bound to a graph
    eval_renderer_.SetStream(stream_);
    return eval_renderer_.Render(gaussians_, camera, options_.background, device_image, sh_degree_);
}

bool GaussianSplatting::Evaluate(const std::vector<CameraParams>& cameras, const std::vector<const uint8_t*>& images,
                                 double* psnr, double* loss) {
    if (!psnr) return false;
    return EvaluateMetrics(cameras, images, psnr, nullptr, nullptr, loss);
}

bool GaussianSplatting::EvaluateMetrics(const std::vector<CameraParams>& cameras,
                                        const std::vector<const uint8_t*>& images, double* psnr, double* ssim,
                                        double* l1, double* loss) {
    if (cameras.size() != images.size() || cameras.empty() || !gaussians_.gaussians_) return false;
    double sums[4] = {0.0, 0.0, 0.0, 0.0};  // PSNR, SSIM, L1 (clamped image), loss
    DeviceArray<uint8_t> target;
    DeviceArray<float> image;
    DeviceArray<double> workspace, metrics;
    Solver objective;
    objective.SetStream(stream_);
    objective.SetComputeLoss(true);
    if (!metrics.Reserve(4)) return false;
    for (size_t k = 0; k < cameras.size(); ++k) {
        const CameraParams& c = cameras[k];
        const size_t px = static_cast<size_t>(c.width_) * c.height_;
        if (!images[k] || !target.Reserve(px * 3) || !image.Reserve(px * 3) ||
            !workspace.Reserve(gsn::eval_metrics_workspace(c.width_, c.height_) / sizeof(double)))
            return false;
        if (cudaMemcpyAsync(target.get(), images[k], px * 3, cudaMemcpyHostToDevice, stream_) != cudaSuccess)
            return false;
        if (!Render(c, image.get()) ||
            gsn::launch_eval_metrics(image.get(), target.get(), c.width_, c.height_, workspace.get(), metrics.get(),
                                     stream_) != GSN_OK)
            return false;
        // the training objective (unclamped image), reduced in FP64 as well
        if (loss && !objective.ComputeImageGradients(c, image.get(), target.get())) return false;
        double m[4], objective_out[4] = {0.0, 0.0, 0.0, 0.0};
        if (cudaMemcpyAsync(m, metrics.get(), sizeof(m), cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
            (loss && cudaMemcpyAsync(objective_out, objective.GetLossDevice(), sizeof(objective_out),
                                     cudaMemcpyDeviceToHost, stream_) != cudaSuccess) ||
            cudaStreamSynchronize(stream_) != cudaSuccess)
            return false;
        sums[0] += m[0];
        sums[1] += m[1];
        sums[2] += m[2];
        sums[3] += objective_out[0];
    }
    const double n = static_cast<double>(cameras.size());
    if (psnr) *psnr = sums[0] / n;
    if (ssim) *ssim = sums[1] / n;
    if (l1) *l1 = sums[2] / n;
    if (loss) *loss = sums[3] / n;
    return true;
}

bool GaussianSplatting::Save(const std::string& path) {
    const int count = gaussians_.gaussian_count_;
    if (count <= 0 || !gaussians_.gaussians_) return false;
    std::vector<float> p;
    if (!GetParameters(p)) return false;
    return WriteGaussiansPly(path, UnpackGaussians(p.data(), count));
}

bool GaussianSplatting::Load(const std::string& path) {
    std::vector<Gaussian> g;
    if (!ReadGaussiansPly(path, g)) return false;
    std::vector<float> p = PackGaussians(g);
    return SetParameters(p.data(), static_cast<int>(g.size()));
}

namespace {

constexpr char kCheckpointMagic[8] = {'G', 'S', 'N', 'C', 'K', 'P', 'T', '1'};
// version 3: the precision layout's SH block holds bf16 pair rows
constexpr uint32_t kCheckpointVersion = 3;

struct CheckpointHeader {
    char magic[8];
    uint32_t version;
    uint32_t bf16_sh;
    int32_t count;
    int32_t rows;
    int32_t completed;
    int32_t sh_degree;
    uint64_t adam_step;
    int32_t camera_cursor;
    int32_t camera_count;
    float scene_extent;
    float scene_centre[3];
};

template <typename T>
bool Download(std::vector<T>& host, const T* device, size_t count) {
    host.resize(count);
    return count == 0 || cudaMemcpy(host.data(), device, count * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess;
}

template <typename T>
bool Upload(T* device, const std::vector<T>& host) {
    return host.empty() || cudaMemcpy(device, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice) ==
                               cudaSuccess;
}

}  // namespace

bool GaussianSplatting::SaveCheckpoint(const std::string& path) {
    const int count = gaussians_.gaussian_count_;
    if (!gaussians_.gaussians_ || count <= 0 || cudaStreamSynchronize(stream_) != cudaSuccess) return false;
    const size_t rows = PhysicalRows(), n = static_cast<size_t>(count);
    CheckpointHeader h{};
    std::memcpy(h.magic, kCheckpointMagic, sizeof(h.magic));
    h.version = kCheckpointVersion;
    h.bf16_sh = options_.bf16_sh ? 1u : 0u;
    h.count = count;
    h.rows = static_cast<int32_t>(rows);
    h.completed = completed_;
    h.sh_degree = sh_degree_;
    h.adam_step = solver_.GetIteration();
    h.camera_cursor = camera_cursor_;
    h.camera_count = static_cast<int32_t>(camera_order_.size());
    h.scene_extent = scene_extent_;
    for (int a = 0; a < 3; ++a) h.scene_centre[a] = scene_centre_[a];
    std::vector<float> block, m, v, sums, abs_sums, max_radius, depth_sum, depth_sq, last_grad;
    std::vector<unsigned int> obs;
    std::vector<int> birth;
    if (!Download(block, gaussians_.gaussians_, rows * n) || !Download(m, solver_.GetFirstMoments(), rows * n) ||
        !Download(v, solver_.GetSecondMoments(), rows * n) ||
        !Download(sums, static_cast<const float*>(density_.GetGradientSums()), n) ||
        !Download(abs_sums, static_cast<const float*>(density_.GetAbsoluteGradientSums()), n) ||
        !Download(obs, static_cast<const unsigned int*>(density_.GetObservationCounts()), n) ||
        !Download(max_radius, static_cast<const float*>(ls_max_radius_.get()), n) ||
        !Download(depth_sum, static_cast<const float*>(ls_depth_sum_.get()), n) ||
        !Download(depth_sq, static_cast<const float*>(ls_depth_sq_.get()), n) ||
        !Download(last_grad, reinterpret_cast<const float*>(ls_last_grad_.get()), 4 * n) ||
        !Download(birth, static_cast<const int*>(ls_birth_.get()), n))
        return false;
    std::ofstream out(path, std::ios::binary);
    if (!out) return false;
    out.write(reinterpret_cast<const char*>(&h), sizeof(h));
    out.write(reinterpret_cast<const char*>(camera_order_.data()), camera_order_.size() * sizeof(int));
    for (const std::vector<float>* a : {&block, &m, &v, &sums, &abs_sums})
        out.write(reinterpret_cast<const char*>(a->data()), a->size() * sizeof(float));
    out.write(reinterpret_cast<const char*>(obs.data()), obs.size() * sizeof(unsigned int));
    // learned-policy statistics (version 2)
    for (const std::vector<float>* a : {&max_radius, &depth_sum, &depth_sq, &last_grad})
        out.write(reinterpret_cast<const char*>(a->data()), a->size() * sizeof(float));
    out.write(reinterpret_cast<const char*>(birth.data()), birth.size() * sizeof(int));
    return static_cast<bool>(out);
}

bool GaussianSplatting::LoadCheckpoint(const std::string& path) {
    if (cameras_.empty()) return false;
    std::ifstream in(path, std::ios::binary);
    CheckpointHeader h{};
    if (!in || !in.read(reinterpret_cast<char*>(&h), sizeof(h)) ||
        std::memcmp(h.magic, kCheckpointMagic, sizeof(h.magic)) != 0 || h.version != kCheckpointVersion ||
        h.bf16_sh != (options_.bf16_sh ? 1u : 0u) || h.count <= 0 || h.rows != static_cast<int32_t>(PhysicalRows()) ||
        h.camera_count != static_cast<int32_t>(cameras_.size()) || h.camera_cursor < 0 ||
        h.camera_cursor > h.camera_count)
        return false;
    const size_t rows = PhysicalRows(), n = static_cast<size_t>(h.count);
    std::vector<int> order(static_cast<size_t>(h.camera_count));
    std::vector<float> block(rows * n), m(rows * n), v(rows * n), sums(n), abs_sums(n);
    std::vector<float> max_radius(n), depth_sum(n), depth_sq(n), last_grad(4 * n);
    std::vector<unsigned int> obs(n);
    std::vector<int> birth(n);
    in.read(reinterpret_cast<char*>(order.data()), order.size() * sizeof(int));
    for (std::vector<float>* a : {&block, &m, &v, &sums, &abs_sums})
        in.read(reinterpret_cast<char*>(a->data()), a->size() * sizeof(float));
    in.read(reinterpret_cast<char*>(obs.data()), obs.size() * sizeof(unsigned int));
    for (std::vector<float>* a : {&max_radius, &depth_sum, &depth_sq, &last_grad})
        in.read(reinterpret_cast<char*>(a->data()), a->size() * sizeof(float));
    in.read(reinterpret_cast<char*>(birth.data()), birth.size() * sizeof(int));
    if (!in) return false;
    for (int k : order)
        if (k < 0 || k >= h.camera_count) return false;
    void* dev = nullptr;
    if (DeviceAlloc(&dev, block.size() * sizeof(float)) != cudaSuccess) return false;
    if (!Upload(static_cast<float*>(dev), block) || !density_.Initialize(h.count, h.count) ||
        !solver_.RemapGaussians(nullptr, h.count)) {
        cudaFree(dev);
        return false;
    }
    graph_.Release();
    cudaFree(gaussians_.gaussians_);
    gaussians_.gaussians_ = static_cast<float*>(dev);
    gaussians_.gaussian_count_ = h.count;
    if (!Upload(solver_.GetFirstMoments(), m) || !Upload(solver_.GetSecondMoments(), v) ||
        !Upload(density_.GetGradientSums(), sums) || !Upload(density_.GetAbsoluteGradientSums(), abs_sums) ||
        !Upload(density_.GetObservationCounts(), obs) || !ResetLearnedStatistics(h.count, nullptr, 0) ||
        cudaStreamSynchronize(stream_) != cudaSuccess ||
        !Upload(ls_max_radius_.get(), max_radius) || !Upload(ls_depth_sum_.get(), depth_sum) ||
        !Upload(ls_depth_sq_.get(), depth_sq) || !Upload(reinterpret_cast<float*>(ls_last_grad_.get()), last_grad) ||
        !Upload(ls_birth_.get(), birth))
        return false;
    solver_.SetIteration(h.adam_step);
    completed_ = h.completed;
    sh_degree_ = h.sh_degree;
    camera_order_ = order;
    camera_cursor_ = h.camera_cursor;
    scene_extent_ = h.scene_extent;
    for (int a = 0; a < 3; ++a) scene_centre_[a] = h.scene_centre[a];
    return cudaDeviceSynchronize() == cudaSuccess;
}

}  // namespace gs_native
