// gs_native::DensityController over the sm_100a kernels of csrc/density.cu
// (reference behaviour: src/core/density/density_controller.cu:312-647).
#include "core/density/density_controller.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <utility>

#include "density.h"
#include "profile.h"

namespace gs_native {

DensityController::~DensityController() {
    cudaFree(spare_gaussian_parameters_);
    cudaFree(history_parent_ids_);
    if (host_control_) cudaFreeHost(host_control_);
}

bool DensityController::Reserve(int capacity) {
    if (capacity <= capacity_ && gradient_sums_.get()) return true;
    const size_t n = static_cast<size_t>(capacity);
    // arrays whose contents must survive the growth: the accumulated statistics
    // and the decisions/offsets of a ControlDensity call in progress
    DeviceArray<float> sums, abs_sums;
    DeviceArray<unsigned int> obs;
    DeviceArray<int4> counts, offsets;
    if (!sums.Reserve(n) || !abs_sums.Reserve(n) || !obs.Reserve(n) || !counts.Reserve(n + 1) ||
        !offsets.Reserve(n + 1))
        return false;
    if (!samples_.Reserve(6 * n) || !parent_ids_.Reserve(n) || !new_flags_.Reserve(n) || !additions_.Reserve(n + 1) ||
        !scan_storage_.Reserve(gsn::density_scan_scratch_bytes(capacity)) ||
        !int_scan_storage_.Reserve(gsn::scan_scratch_bytes(capacity)))
        return false;
    const size_t old = gradient_sums_.get() ? static_cast<size_t>(capacity_) : 0;
    if (old > 0) {
        if (cudaMemcpyAsync(sums.get(), gradient_sums_.get(), old * sizeof(float), cudaMemcpyDeviceToDevice,
                            stream_) != cudaSuccess ||
            cudaMemcpyAsync(abs_sums.get(), absolute_gradient_sums_.get(), old * sizeof(float),
                            cudaMemcpyDeviceToDevice, stream_) != cudaSuccess ||
            cudaMemcpyAsync(obs.get(), observation_counts_.get(), old * sizeof(unsigned int),
                            cudaMemcpyDeviceToDevice, stream_) != cudaSuccess ||
            cudaMemcpyAsync(counts.get(), density_counts_.get(), (old + 1) * sizeof(int4), cudaMemcpyDeviceToDevice,
                            stream_) != cudaSuccess ||
            cudaMemcpyAsync(offsets.get(), density_offsets_.get(), (old + 1) * sizeof(int4),
                            cudaMemcpyDeviceToDevice, stream_) != cudaSuccess)
            return false;
    }
    if (cudaMemsetAsync(sums.get() + old, 0, (n - old) * sizeof(float), stream_) != cudaSuccess ||
        cudaMemsetAsync(abs_sums.get() + old, 0, (n - old) * sizeof(float), stream_) != cudaSuccess ||
        cudaMemsetAsync(obs.get() + old, 0, (n - old) * sizeof(unsigned int), stream_) != cudaSuccess)
        return false;
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return false;
    gradient_sums_ = std::move(sums);
    absolute_gradient_sums_ = std::move(abs_sums);
    observation_counts_ = std::move(obs);
    density_counts_ = std::move(counts);
    density_offsets_ = std::move(offsets);
    capacity_ = capacity;
    return true;
}

bool DensityController::Initialize(int gaussian_count, int capacity) {
    if (gaussian_count < 0 || capacity < gaussian_count || capacity < 0 || capacity > INT_MAX / 6) return false;
    if (!control_.get() && !control_.Reserve((gsn::kDensityControlBytes + sizeof(int) - 1) / sizeof(int))) return false;
    if (!host_control_ && cudaMallocHost(&host_control_, 8 * sizeof(int)) != cudaSuccess) {
        host_control_ = nullptr;
        return false;
    }
    if (!Reserve(std::max(capacity, 1))) return false;
    if (cudaMemsetAsync(gradient_sums_.get(), 0, sizeof(float) * capacity_, stream_) != cudaSuccess ||
        cudaMemsetAsync(absolute_gradient_sums_.get(), 0, sizeof(float) * capacity_, stream_) != cudaSuccess ||
        cudaMemsetAsync(observation_counts_.get(), 0, sizeof(unsigned int) * capacity_, stream_) != cudaSuccess)
        return false;
    int device = 0, sms = 0, threads_per_sm = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&threads_per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device) != cudaSuccess)
        return false;
    random_blocks_ = std::max(1, sms * (threads_per_sm / 256));
    if (gsn::launch_density_init(control_.get(), gaussian_count, stream_) != GSN_OK) return false;
    parameter_stride_ = capacity;
    seed_ = 0;
    return true;
}

bool DensityController::AccumulateStatistics(const float* gradients, const float* radii, const int* gaussian_ids,
                                             int observation_count) {
    if (observation_count == 0) return true;
    if (!control_.get() || !gradients || !radii || observation_count < 0) return false;
    return gsn::launch_density_accumulate_observations(gradients, radii, gaussian_ids, control_.get(),
                                                       gradient_sums_.get(), observation_counts_.get(),
                                                       observation_count, stream_) == GSN_OK;
}

bool DensityController::AccumulateStatistics(const float* statistics, const float* absolute_statistics,
                                             int gaussian_count) {
    if (gaussian_count == 0) return true;
    if (!control_.get() || !statistics || !absolute_statistics || gaussian_count < 0 || gaussian_count > capacity_)
        return false;
    return gsn::launch_density_accumulate(statistics, absolute_statistics, control_.get(), gradient_sums_.get(),
                                          absolute_gradient_sums_.get(), observation_counts_.get(), gaussian_count,
                                          stream_) == GSN_OK;
}

bool DensityController::ResetOpacity(float* parameters, int stride, float max_opacity) {
    if (!control_.get() || stride != parameter_stride_ || (!parameters && stride > 0) || !std::isfinite(max_opacity) ||
        max_opacity <= 0.0f || max_opacity >= 1.0f)
        return false;
    const float max_logit = std::log(max_opacity / (1.0f - max_opacity));
    return gsn::launch_density_reset_opacity(control_.get(), parameters, stride, max_logit, stream_) == GSN_OK;
}

bool DensityController::ControlDensity(GaussianBuffers& gaussians, float scene_extent, float gradient_threshold,
                                       float percent_dense, float min_opacity, float max_screen_size,
                                       unsigned long long seed, int* changes, float absolute_gradient_threshold) {
    const int count = gaussians.gaussian_count_;
    const float* params = gaussians.gaussians_;
    if (!control_.get() || (!params && count > 0) || (params && params == spare_gaussian_parameters_) || count < 0 ||
        count != parameter_stride_ || spare_gaussian_stride_ < 0 || spare_gaussian_stride_ > INT_MAX / 6 ||
        !std::isfinite(scene_extent) || scene_extent < 0 || !std::isfinite(gradient_threshold) ||
        gradient_threshold < 0 || !std::isfinite(percent_dense) || percent_dense < 0 || !std::isfinite(min_opacity) ||
        min_opacity < 0 || min_opacity > 1 || !std::isfinite(max_screen_size) || max_screen_size < 0 ||
        !std::isfinite(absolute_gradient_threshold) || absolute_gradient_threshold < 0)
        return false;
    if (!Reserve(std::max(count, 1))) return false;
    gsn::stage_mark(stream_, gsn::kStageDensity);
    gsn::DensityDecideArgs d{};
    d.params = params;
    d.sums = gradient_sums_.get();
    d.abs_sums = absolute_gradient_sums_.get();
    d.obs = observation_counts_.get();
    d.control = control_.get();
    d.counts = density_counts_.get();
    d.offsets = density_offsets_.get();
    d.scan_scratch = reinterpret_cast<int4*>(scan_storage_.get());
    d.additions = additions_.get();
    d.int_scan_scratch = int_scan_storage_.get();
    d.n = count;
    d.max_count = max_gaussians_;
    d.random_blocks = random_blocks_;
    d.th.gradient_threshold = gradient_threshold;
    d.th.split_threshold = percent_dense * scene_extent;
    d.th.min_opacity = min_opacity;
    d.th.max_world_size = 0.1f * scene_extent;
    d.th.absolute_gradient_threshold = absolute_gradient_threshold;
    d.th.prune_large = max_screen_size > 0;
    d.actions = actions_;
    if (gsn::launch_density_decide(d, stream_) != GSN_OK) return false;
    if (cudaMemcpyAsync(host_control_, control_.get(), 8 * sizeof(int), cudaMemcpyDeviceToHost, stream_) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
        return false;
    const int required = host_control_[1];
    if (changes) {
        changes[0] = host_control_[5] + 2 * host_control_[6];
        changes[1] = host_control_[7] - host_control_[4];
    }
    const int next_stride = required;
    if (!Reserve(std::max(count, std::max(next_stride, spare_gaussian_stride_)))) return false;
    if (required == 0) {
        cudaFree(spare_gaussian_parameters_);
        cudaFree(history_parent_ids_);
        spare_gaussian_parameters_ = nullptr;
        history_parent_ids_ = nullptr;
        spare_gaussian_stride_ = 0;
    } else if (!spare_gaussian_parameters_ || next_stride > spare_gaussian_stride_) {
        void* replacement = nullptr;
        const size_t rows = bf16_sh_ ? 34 : kMaxParamCount;
        if (DeviceAlloc(&replacement, sizeof(float) * rows * static_cast<size_t>(next_stride)) != cudaSuccess)
            return false;
        cudaFree(spare_gaussian_parameters_);
        spare_gaussian_parameters_ = static_cast<float*>(replacement);
        spare_gaussian_stride_ = next_stride;
    }
    if (required > 0) {
        void* hp = nullptr;
        if (DeviceAlloc(&hp, static_cast<size_t>(required) * sizeof(int)) != cudaSuccess) return false;
        cudaFree(history_parent_ids_);
        history_parent_ids_ = static_cast<int*>(hp);
    }
    spare_gaussian_stride_ = next_stride;
    if (seed != seed_) {
        if (cudaMemsetAsync(control_.get() + 8, 0, 2 * sizeof(unsigned long long), stream_) != cudaSuccess)
            return false;
        seed_ = seed;
        if (gsn::launch_density_prepare(density_offsets_.get(), control_.get(), count, random_blocks_, stream_) !=
            GSN_OK)
            return false;
    }
    gsn::DensityApplyArgs a{};
    a.params = params;
    a.counts = density_counts_.get();
    a.offsets = density_offsets_.get();
    a.control = control_.get();
    a.samples = samples_.get();
    a.out = spare_gaussian_parameters_;
    a.history_parents = history_parent_ids_;
    a.parents = parent_ids_.get();
    a.new_flags = new_flags_.get();
    a.sums = gradient_sums_.get();
    a.abs_sums = absolute_gradient_sums_.get();
    a.obs = observation_counts_.get();
    a.n = count;
    a.out_stride = spare_gaussian_stride_;
    a.random_blocks = random_blocks_;
    a.seed = seed;
    a.bf16_sh = bf16_sh_;
    if (gsn::launch_density_apply(a, stream_) != GSN_OK) return false;
    gsn::stage_mark(stream_, gsn::kStageOther);
    parameter_stride_ = next_stride;
    std::swap(gaussians.gaussians_, spare_gaussian_parameters_);
    gaussians.gaussian_count_ = next_stride;
    spare_gaussian_stride_ = count;
    return true;
}

bool DensityController::GetDecisionCodes(int8_t* codes, int count) const {
    if (!codes || count < 0 || count > capacity_ || !density_counts_.get()) return false;
    return gsn::launch_density_codes(density_counts_.get(), count, codes, stream_) == GSN_OK;
}

bool DensityController::ComputeFeatures(const GaussianBuffers& gaussians, float scene_extent,
                                        float gradient_threshold, float percent_dense,
                                        const gsn::LearnedStatsView& ls, float* features) const {
    const int count = gaussians.gaussian_count_;
    if (count == 0) return true;
    if (!features || !gaussians.gaussians_ || count < 0 || count > capacity_ || !gradient_sums_.get()) return false;
    gsn::DensityThresholds th{};
    th.gradient_threshold = gradient_threshold;
    th.split_threshold = percent_dense * scene_extent;
    return gsn::launch_density_features(gaussians.gaussians_, gradient_sums_.get(), observation_counts_.get(), count,
                                        th, scene_extent, ls, bf16_sh_, features, stream_) == GSN_OK;
}

}  // namespace gs_native
