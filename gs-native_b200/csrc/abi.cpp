// extern "C" ABI of the gs-native B200 library (declarations in include/gsn.h).
#include "gsn.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "core/density/density_controller.h"
#include "core/density/density_mlp.h"
#include "core/gaussian_splatting.h"
#include "core/graph/training_graph.h"
#include "io/colmap.h"
#include "io/image.h"
#include "io/ply.h"
#include "core/knn/knn.h"
#include "core/render/multiview_renderer.h"
#include "core/render/renderer.h"
#include "core/solver/solver.h"
#include "core/spatial/spatial_order.h"
#include "kernels.h"
#include "knn_kernels.h"
#include "profile.h"

struct gsn_renderer {
    gs_native::Renderer impl;
};

struct gsn_solver {
    gs_native::Solver impl;
};

struct gsn_density {
    gs_native::DensityController impl;
};

struct gsn_trainer {
    gs_native::GaussianSplatting impl;
};

struct gsn_multiview {
    gs_native::MultiViewRenderer impl;
};

struct gsn_mlp {
    gs_native::DensityMlp impl;
};

struct gsn_graph {
    gs_native::TrainingGraph impl;
    gs_native::GaussianBuffers gaussians;
};

namespace {

inline cudaStream_t AsStream(void* s) { return static_cast<cudaStream_t>(s); }

inline const gs_native::CameraParams& AsCamera(const gsn_camera* c) {
    return *reinterpret_cast<const gs_native::CameraParams*>(c);
}

inline gs_native::GaussianBuffers View(const float* params, int count) {
    gs_native::GaussianBuffers g;
    g.gaussians_ = const_cast<float*>(params);
    g.gaussian_count_ = count;
    return g;
}

}  // namespace

extern "C" {

const char* gsn_version(void) { return "gs-native-b200 0.1.0 (sm_100a)"; }

int gsn_memcpy(void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return GSN_OK;
    if (!dst || !src) return GSN_ERR_INVALID_ARGUMENT;
    return cudaMemcpy(dst, src, bytes, cudaMemcpyDefault) == cudaSuccess ? GSN_OK : GSN_ERR_CUDA;
}

int gsn_memcpy_async(void* dst, const void* src, size_t bytes, void* stream) {
    if (bytes == 0) return GSN_OK;
    if (!dst || !src) return GSN_ERR_INVALID_ARGUMENT;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, AsStream(stream)) == cudaSuccess ? GSN_OK
                                                                                               : GSN_ERR_CUDA;
}

int gsn_device_alloc(size_t bytes, void** out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (bytes == 0) return GSN_OK;
    return cudaMalloc(out, bytes) == cudaSuccess ? GSN_OK : GSN_ERR_OUT_OF_MEMORY;
}

int gsn_device_free(void* ptr) { return cudaFree(ptr) == cudaSuccess ? GSN_OK : GSN_ERR_CUDA; }

int gsn_stream_synchronize(void* stream) {
    return cudaStreamSynchronize(AsStream(stream)) == cudaSuccess ? GSN_OK : GSN_ERR_CUDA;
}

uint64_t gsn_kernel_launch_count(void) { return gsn::launch_count(); }

int gsn_set_programmatic_launch(int enabled) {
    gsn::set_programmatic_launch(enabled != 0);
    return GSN_OK;
}

int gsn_profile_enable(int enabled) {
    gsn::profile_enable(enabled != 0);
    return GSN_OK;
}

int gsn_profile_collect(double* ms, int count) {
    if (!ms || count < 0) return GSN_ERR_INVALID_ARGUMENT;
    return gsn::profile_collect(ms, count) == 0 ? GSN_OK : GSN_ERR_CUDA;
}

const char* gsn_stage_name(int stage) { return gsn::stage_name(stage); }

int gsn_stage_count(void) { return gsn::kStageCount; }

int gsn_sort_pairs_workspace(int max_count, size_t* bytes) {
    if (!bytes || max_count < 0) return GSN_ERR_INVALID_ARGUMENT;
    *bytes = gsn::radix_sort_scratch_bytes(max_count);
    return GSN_OK;
}

int gsn_sort_pairs(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt, int count,
                   int begin_bit, int end_bit, void* workspace, size_t workspace_bytes, int* result_in_alt,
                   void* stream) {
    if (!result_in_alt || count < 0 || begin_bit < 0 || end_bit > 32 || end_bit < begin_bit) return GSN_ERR_INVALID_ARGUMENT;
    *result_in_alt = 0;
    if (count == 0 || end_bit == begin_bit) return GSN_OK;
    if (!keys || !values || !keys_alt || !values_alt || !workspace ||
        workspace_bytes < gsn::radix_sort_scratch_bytes(count))
        return GSN_ERR_INVALID_ARGUMENT;
    gsn::RadixSortScratch scratch = gsn::radix_sort_scratch(workspace, count);
    bool alt = false;
    int status = gsn::launch_radix_sort(keys, values, keys_alt, values_alt, false, count, nullptr, begin_bit, end_bit,
                                        scratch, &alt, AsStream(stream));
    *result_in_alt = alt ? 1 : 0;
    return status;
}

int gsn_exclusive_scan_workspace(int max_count, size_t* bytes) {
    if (!bytes || max_count < 0) return GSN_ERR_INVALID_ARGUMENT;
    *bytes = gsn::scan_scratch_bytes(max_count);
    return GSN_OK;
}

int gsn_exclusive_scan(const int* in, const uint32_t* gather, int* out, int count, const int* valid,
                       void* workspace, size_t workspace_bytes, void* stream) {
    if (count < 0 || !out || (count > 0 && (!in || !workspace || workspace_bytes < gsn::scan_scratch_bytes(count))))
        return GSN_ERR_INVALID_ARGUMENT;
    return gsn::launch_exclusive_scan(in, gather, out, count, workspace, AsStream(stream), valid);
}

int gsn_sort_pairs_noalloc(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt, int count,
                           int begin_bit, int end_bit, int* result_in_alt, void* stream) {
    if (!result_in_alt || count < 0 || begin_bit < 0 || end_bit > 32 || end_bit < begin_bit) return GSN_ERR_INVALID_ARGUMENT;
    *result_in_alt = 0;
    if (count > gsn::noalloc_sort_max_count()) return GSN_ERR_CAPACITY;
    if (count == 0 || end_bit == begin_bit) return GSN_OK;
    if (!keys || !values || !keys_alt || !values_alt) return GSN_ERR_INVALID_ARGUMENT;
    bool alt = false;
    int status = gsn::launch_radix_sort_noalloc(keys, values, keys_alt, values_alt, count, begin_bit, end_bit, &alt,
                                                AsStream(stream));
    *result_in_alt = alt ? 1 : 0;
    return status;
}

int gsn_knn3_workspace(int count, size_t* bytes) {
    if (!bytes || count < 0) return GSN_ERR_INVALID_ARGUMENT;
    *bytes = gsn::knn_layout(count).total;
    return GSN_OK;
}

int gsn_knn3(const float* points, int count, float* mean_dist2, int* neighbors, void* workspace, void* stream) {
    if (count < 0 || (count > 0 && (!points || !mean_dist2 || !workspace))) return GSN_ERR_INVALID_ARGUMENT;
    return gsn::launch_knn3(points, count, mean_dist2, neighbors, workspace, AsStream(stream));
}

int gsn_knn3_host(const float* points, int count, float* mean_dist2, int* neighbors) {
    return gs_native::ComputeMeanDist2(points, count, mean_dist2, neighbors) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_renderer_create(gsn_renderer** out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    *out = new (std::nothrow) gsn_renderer();
    return *out ? GSN_OK : GSN_ERR_OUT_OF_MEMORY;
}

int gsn_renderer_destroy(gsn_renderer* r) {
    delete r;
    return GSN_OK;
}

int gsn_renderer_set_stream(gsn_renderer* r, void* stream) {
    if (!r) return GSN_ERR_INVALID_ARGUMENT;
    r->impl.SetStream(AsStream(stream));
    return GSN_OK;
}

int gsn_renderer_render(gsn_renderer* r, const float* params, int count, const gsn_camera* camera,
                        const float* background, float* image, int sh_degree) {
    if (!r || !camera) return GSN_ERR_INVALID_ARGUMENT;
    gs_native::GaussianBuffers g;
    g.gaussians_ = const_cast<float*>(params);
    g.gaussian_count_ = count;
    const auto& cam = *reinterpret_cast<const gs_native::CameraParams*>(camera);
    return r->impl.Render(g, cam, background, image, sh_degree) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_renderer_get_buffers(gsn_renderer* r, gsn_renderer_buffers* out) {
    if (!r || !out) return GSN_ERR_INVALID_ARGUMENT;
    const auto& R = r->impl;
    out->means = reinterpret_cast<const float*>(R.GetMeans());
    out->conic_opacity = reinterpret_cast<const float*>(R.GetConicOpacities());
    out->colors = reinterpret_cast<const float*>(R.GetColors());
    out->depths = R.GetDepths();
    out->rects = reinterpret_cast<const int*>(R.GetTileRects());
    out->tile_counts = R.GetTileCounts();
    out->radii = R.GetRadii();
    out->tile_gaussian_ids = R.GetTileGaussianIds();
    out->tile_offsets = R.GetTileGaussianOffsets();
    out->contributors = R.GetContributors();
    out->record_count = R.GetRecordCountDevice();
    out->overflow = R.GetOverflowFlag();
    out->record_count_host = R.GetLastRecordCount();
    out->gaussian_capacity = R.GetGaussianCapacity();
    out->tile_capacity = R.GetTileCapacity();
    return GSN_OK;
}

int gsn_renderer_record_offsets(gsn_renderer* r, const int** out) {
    if (!r || !out) return GSN_ERR_INVALID_ARGUMENT;
    *out = r->impl.GetRecordOffsets();
    return *out ? GSN_OK : GSN_ERR_CUDA;
}

int gsn_renderer_set_bf16_sh(gsn_renderer* r, int enabled) {
    if (!r) return GSN_ERR_INVALID_ARGUMENT;
    r->impl.SetBf16Sh(enabled != 0);
    return GSN_OK;
}

int gsn_renderer_set_exact_culling(gsn_renderer* r, int enabled) {
    if (!r) return GSN_ERR_INVALID_ARGUMENT;
    r->impl.SetExactCulling(enabled != 0);
    return GSN_OK;
}

int gsn_renderer_set_fast_blend(gsn_renderer* r, int enabled) {
    if (!r) return GSN_ERR_INVALID_ARGUMENT;
    r->impl.SetFastBlend(enabled != 0);
    return GSN_OK;
}

int gsn_renderer_set_pair_counter(gsn_renderer* r, unsigned long long* device_counter) {
    if (!r) return GSN_ERR_INVALID_ARGUMENT;
    r->impl.SetPairCounter(device_counter);
    return GSN_OK;
}

int gsn_renderer_set_record_capacity(gsn_renderer* r, int64_t records) {
    if (!r) return GSN_ERR_INVALID_ARGUMENT;
    return r->impl.SetRecordCapacity(records) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_solver_create(gsn_solver** out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    *out = new (std::nothrow) gsn_solver();
    return *out ? GSN_OK : GSN_ERR_OUT_OF_MEMORY;
}

int gsn_solver_destroy(gsn_solver* s) {
    delete s;
    return GSN_OK;
}

int gsn_solver_set_stream(gsn_solver* s, void* stream) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    s->impl.SetStream(AsStream(stream));
    return GSN_OK;
}

int gsn_solver_iterate(gsn_solver* s, const gsn_camera* camera, gsn_renderer* renderer, const float* image,
                       const uint8_t* target, float* params, int count, float position_lr, int sh_degree) {
    if (!s || !camera || !renderer) return GSN_ERR_INVALID_ARGUMENT;
    gs_native::GaussianBuffers g = View(params, count);
    return s->impl.Iterate(AsCamera(camera), renderer->impl, image, target, g, position_lr, sh_degree)
               ? GSN_OK
               : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_solver_reset_opacity_history(gsn_solver* s) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    return s->impl.ResetOpacityHistory() ? GSN_OK : GSN_ERR_CUDA;
}

int gsn_solver_remap(gsn_solver* s, const int* parent_ids, int count) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    return s->impl.RemapGaussians(parent_ids, count) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_solver_statistics(gsn_solver* s, const float** stats, const float** absolute_stats) {
    if (!s || !stats || !absolute_stats) return GSN_ERR_INVALID_ARGUMENT;
    *stats = s->impl.GetProjectionStatistics();
    *absolute_stats = s->impl.GetAbsoluteProjectionStatistics();
    return GSN_OK;
}

int gsn_solver_set_learning_rates(gsn_solver* s, float scale, float rotation, float opacity, float sh_dc,
                                  float sh_rest) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    gs_native::LearningRates lr;
    lr.scale = scale;
    lr.rotation = rotation;
    lr.opacity = opacity;
    lr.sh_dc = sh_dc;
    lr.sh_rest = sh_rest;
    s->impl.SetLearningRates(lr);
    return GSN_OK;
}

int gsn_solver_set_bf16_sh(gsn_solver* s, int enabled) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    s->impl.SetBf16Sh(enabled != 0);
    return GSN_OK;
}

int gsn_solver_set_tensor_core_loss(gsn_solver* s, int enabled) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    s->impl.SetTensorCoreLoss(enabled != 0);
    return GSN_OK;
}

int gsn_solver_set_sparse_adam(gsn_solver* s, int enabled) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    s->impl.SetSparseAdam(enabled != 0);
    return GSN_OK;
}

int gsn_solver_set_lazy_moment_decay(gsn_solver* s, int enabled) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    s->impl.SetLazyMomentDecay(enabled != 0);
    return GSN_OK;
}

int gsn_solver_status(gsn_solver* s, int* status) {
    if (!s || !status) return GSN_ERR_INVALID_ARGUMENT;
    *status = GSN_OK;
    if (!s->impl.GetStatusDevice()) return GSN_OK;
    return cudaMemcpy(status, s->impl.GetStatusDevice(), sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess
               ? GSN_OK
               : GSN_ERR_CUDA;
}

int gsn_solver_set_compute_loss(gsn_solver* s, int enabled) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    s->impl.SetComputeLoss(enabled != 0);
    return GSN_OK;
}

int gsn_solver_loss(gsn_solver* s, double* out) {
    if (!s || !out || !s->impl.GetLossDevice()) return GSN_ERR_INVALID_ARGUMENT;
    return cudaMemcpy(out, s->impl.GetLossDevice(), 4 * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess
               ? GSN_OK
               : GSN_ERR_CUDA;
}

int gsn_solver_loss_device(gsn_solver* s, const double** out) {
    if (!s || !out) return GSN_ERR_INVALID_ARGUMENT;
    *out = s->impl.GetLossDevice();
    return *out ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_solver_image_gradients(gsn_solver* s, const gsn_camera* camera, const float* image, const uint8_t* target,
                               const float** out) {
    if (!s || !camera || !out) return GSN_ERR_INVALID_ARGUMENT;
    if (!s->impl.ComputeImageGradients(AsCamera(camera), image, target)) return GSN_ERR_INVALID_ARGUMENT;
    *out = s->impl.GetImageGradients();
    return GSN_OK;
}

int gsn_solver_screen_gradients(gsn_solver* s, const gsn_camera* camera, gsn_renderer* renderer,
                                const float* image, const float* params, int count, const float** out) {
    if (!s || !camera || !renderer || !out) return GSN_ERR_INVALID_ARGUMENT;
    if (!s->impl.ComputeScreenGradients(AsCamera(camera), renderer->impl, View(params, count), image))
        return GSN_ERR_INVALID_ARGUMENT;
    *out = s->impl.GetScreenGradients();
    return GSN_OK;
}

int gsn_solver_map_gradients(gsn_solver* s, const gsn_camera* camera, gsn_renderer* renderer, float* params,
                             int count, int sh_degree, float* grads_out) {
    if (!s || !camera || !renderer || !grads_out) return GSN_ERR_INVALID_ARGUMENT;
    gs_native::GaussianBuffers g = View(params, count);
    return s->impl.UpdateGaussians(AsCamera(camera), renderer->impl, g, 0.0f, sh_degree, false, grads_out)
               ? GSN_OK
               : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_solver_moments(gsn_solver* s, float** first, float** second, uint64_t* iteration) {
    if (!s || !first || !second || !iteration) return GSN_ERR_INVALID_ARGUMENT;
    *first = s->impl.GetFirstMoments();
    *second = s->impl.GetSecondMoments();
    *iteration = s->impl.GetIteration();
    return GSN_OK;
}

int gsn_density_create(gsn_density** out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    *out = new (std::nothrow) gsn_density();
    return *out ? GSN_OK : GSN_ERR_OUT_OF_MEMORY;
}

int gsn_density_destroy(gsn_density* d) {
    delete d;
    return GSN_OK;
}

int gsn_density_set_stream(gsn_density* d, void* stream) {
    if (!d) return GSN_ERR_INVALID_ARGUMENT;
    d->impl.SetStream(AsStream(stream));
    return GSN_OK;
}

int gsn_density_initialize(gsn_density* d, int count, int capacity) {
    if (!d) return GSN_ERR_INVALID_ARGUMENT;
    return d->impl.Initialize(count, capacity) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_density_accumulate(gsn_density* d, const float* statistics, const float* absolute_statistics, int count) {
    if (!d) return GSN_ERR_INVALID_ARGUMENT;
    return d->impl.AccumulateStatistics(statistics, absolute_statistics, count) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_density_accumulate_observations(gsn_density* d, const float* gradients, const float* radii, const int* ids,
                                        int observations) {
    if (!d) return GSN_ERR_INVALID_ARGUMENT;
    return d->impl.AccumulateStatistics(gradients, radii, ids, observations) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_density_reset_opacity(gsn_density* d, float* params, int stride, float max_opacity) {
    if (!d) return GSN_ERR_INVALID_ARGUMENT;
    return d->impl.ResetOpacity(params, stride, max_opacity) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_density_control(gsn_density* d, float** params, int* count, float scene_extent, float gradient_threshold,
                        float percent_dense, float min_opacity, float max_screen_size, unsigned long long seed,
                        int* changes, float absolute_gradient_threshold) {
    if (!d || !params || !count) return GSN_ERR_INVALID_ARGUMENT;
    gs_native::GaussianBuffers g;
    g.gaussians_ = *params;
    g.gaussian_count_ = *count;
    if (!d->impl.ControlDensity(g, scene_extent, gradient_threshold, percent_dense, min_opacity, max_screen_size, seed,
                                changes, absolute_gradient_threshold))
        return GSN_ERR_INVALID_ARGUMENT;
    *params = g.gaussians_;
    *count = g.gaussian_count_;
    return GSN_OK;
}

int gsn_density_buffers(gsn_density* d, const int** history_parent_ids, const int** control, const int** parent_ids) {
    if (!d || !history_parent_ids || !control || !parent_ids) return GSN_ERR_INVALID_ARGUMENT;
    *history_parent_ids = d->impl.GetHistoryParentIds();
    *control = d->impl.GetGaussianCount();
    *parent_ids = d->impl.GetParentIds();
    return GSN_OK;
}

int gsn_density_set_bf16_sh(gsn_density* d, int enabled) {
    if (!d) return GSN_ERR_INVALID_ARGUMENT;
    d->impl.SetBf16Sh(enabled != 0);
    return GSN_OK;
}

int gsn_density_set_max_gaussians(gsn_density* d, int max_gaussians) {
    if (!d || max_gaussians < 0) return GSN_ERR_INVALID_ARGUMENT;
    d->impl.SetMaxGaussians(max_gaussians);
    return GSN_OK;
}

int gsn_density_internals(gsn_density* d, const float** samples, float** gradient_sums, float** absolute_sums,
                          unsigned int** observation_counts) {
    if (!d || !samples || !gradient_sums || !absolute_sums || !observation_counts) return GSN_ERR_INVALID_ARGUMENT;
    *samples = d->impl.GetSamples();
    *gradient_sums = d->impl.GetGradientSums();
    *absolute_sums = d->impl.GetAbsoluteGradientSums();
    *observation_counts = d->impl.GetObservationCounts();
    return GSN_OK;
}

int gsn_training_options_default(gsn_training_options* out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    gs_native::TrainingOptions o;
    out->sh_degree_interval = o.sh_degree_interval;
    out->max_sh_degree = o.max_sh_degree;
    out->position_lr_init = o.position_lr_init;
    out->position_lr_final = o.position_lr_final;
    out->position_lr_steps = o.position_lr_steps;
    out->lr_scale = o.lr.scale;
    out->lr_rotation = o.lr.rotation;
    out->lr_opacity = o.lr.opacity;
    out->lr_sh_dc = o.lr.sh_dc;
    out->lr_sh_rest = o.lr.sh_rest;
    out->densify_from = o.densify_from;
    out->densify_until = o.densify_until;
    out->densify_interval = o.densify_interval;
    out->gradient_threshold = o.gradient_threshold;
    out->absolute_gradient_threshold = o.absolute_gradient_threshold;
    out->percent_dense = o.percent_dense;
    out->min_opacity = o.min_opacity;
    out->prune_large_after = o.prune_large_after;
    out->opacity_cap_interval = o.opacity_cap_interval;
    out->opacity_cap = o.opacity_cap;
    out->opacity_reset_interval = o.opacity_reset_interval;
    out->opacity_reset = o.opacity_reset;
    for (int c = 0; c < 3; ++c) out->background[c] = o.background[c];
    out->max_gaussians = o.max_gaussians;
    out->density_seed = o.density_seed;
    out->initial_opacity = o.initial_opacity;
    out->precision = o.bf16_sh ? 1 : 0;
    out->graph = o.graph ? 1 : 0;
    out->learned_density = o.learned_density ? 1 : 0;
    out->learned_confidence = o.learned_confidence;
    out->log_density = o.log_density ? 1 : 0;
    out->exact_culling = o.exact_culling ? 1 : 0;
    out->sparse_adam = o.sparse_adam ? 1 : 0;
    out->spatial_order = o.spatial_order ? 1 : 0;
    out->fast_blend = o.fast_blend ? 1 : 0;
    out->fp32_ssim = o.fp32_ssim ? 1 : 0;
    return GSN_OK;
}

namespace {
gs_native::TrainingOptions ToOptions(const gsn_training_options& in) {
    gs_native::TrainingOptions o;
    o.sh_degree_interval = in.sh_degree_interval;
    o.max_sh_degree = in.max_sh_degree;
    o.position_lr_init = in.position_lr_init;
    o.position_lr_final = in.position_lr_final;
    o.position_lr_steps = in.position_lr_steps;
    o.lr.scale = in.lr_scale;
    o.lr.rotation = in.lr_rotation;
    o.lr.opacity = in.lr_opacity;
    o.lr.sh_dc = in.lr_sh_dc;
    o.lr.sh_rest = in.lr_sh_rest;
    o.densify_from = in.densify_from;
    o.densify_until = in.densify_until;
    o.densify_interval = in.densify_interval;
    o.gradient_threshold = in.gradient_threshold;
    o.absolute_gradient_threshold = in.absolute_gradient_threshold;
    o.percent_dense = in.percent_dense;
    o.min_opacity = in.min_opacity;
    o.prune_large_after = in.prune_large_after;
    o.opacity_cap_interval = in.opacity_cap_interval;
    o.opacity_cap = in.opacity_cap;
    o.opacity_reset_interval = in.opacity_reset_interval;
    o.opacity_reset = in.opacity_reset;
    for (int c = 0; c < 3; ++c) o.background[c] = in.background[c];
    o.max_gaussians = in.max_gaussians;
    o.density_seed = in.density_seed;
    o.initial_opacity = in.initial_opacity;
    o.bf16_sh = in.precision != 0;
    o.graph = in.graph != 0;
    o.learned_density = in.learned_density != 0;
    o.learned_confidence = in.learned_confidence;
    o.log_density = in.log_density != 0;
    o.exact_culling = in.exact_culling != 0;
    o.sparse_adam = in.sparse_adam != 0;
    o.spatial_order = in.spatial_order != 0;
    o.fast_blend = in.fast_blend != 0;
    o.fp32_ssim = in.fp32_ssim != 0;
    return o;
}
}  // namespace

int gsn_trainer_create(gsn_trainer** out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    *out = new (std::nothrow) gsn_trainer();
    return *out ? GSN_OK : GSN_ERR_OUT_OF_MEMORY;
}

int gsn_trainer_destroy(gsn_trainer* t) {
    delete t;
    return GSN_OK;
}

int gsn_trainer_set_stream(gsn_trainer* t, void* stream) {
    if (!t) return GSN_ERR_INVALID_ARGUMENT;
    t->impl.SetStream(AsStream(stream));
    return GSN_OK;
}

int gsn_trainer_set_lazy_moment_decay(gsn_trainer* t, int enabled) {
    if (!t) return GSN_ERR_INVALID_ARGUMENT;
    t->impl.GetSolver().SetLazyMomentDecay(enabled != 0);
    return GSN_OK;
}

int gsn_trainer_initialize(gsn_trainer* t, const gsn_camera* cameras, const uint8_t* const* images,
                           int camera_count, const float* points, const float* colors, int point_count,
                           const gsn_training_options* options) {
    if (!t || !cameras || !images || camera_count <= 0 || !points || !colors || point_count <= 0)
        return GSN_ERR_INVALID_ARGUMENT;
    gs_native::TrainingScene scene;
    for (int k = 0; k < camera_count; ++k) {
        scene.train_cameras.push_back(AsCamera(cameras + k));
        scene.train_images.push_back(images[k]);
    }
    scene.point_positions = points;
    scene.point_colors = colors;
    scene.point_count = point_count;
    gs_native::TrainingOptions o;
    if (options) o = ToOptions(*options);
    return t->impl.Initialize(scene, o) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_trainer_train(gsn_trainer* t, int iterations) {
    if (!t) return GSN_ERR_INVALID_ARGUMENT;
    return t->impl.Train(iterations) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_trainer_render(gsn_trainer* t, const gsn_camera* camera, float* image) {
    if (!t || !camera) return GSN_ERR_INVALID_ARGUMENT;
    return t->impl.Render(AsCamera(camera), image) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_trainer_evaluate(gsn_trainer* t, const gsn_camera* cameras, const uint8_t* const* images, int count,
                         double* psnr, double* loss) {
    if (!t || !cameras || !images || count <= 0 || !psnr) return GSN_ERR_INVALID_ARGUMENT;
    std::vector<gs_native::CameraParams> cams;
    std::vector<const uint8_t*> imgs;
    for (int k = 0; k < count; ++k) {
        cams.push_back(AsCamera(cameras + k));
        imgs.push_back(images[k]);
    }
    return t->impl.Evaluate(cams, imgs, psnr, loss) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_trainer_evaluate_metrics(gsn_trainer* t, const gsn_camera* cameras, const uint8_t* const* images, int count,
                                 double* psnr, double* ssim, double* l1, double* loss) {
    if (!t || !cameras || !images || count <= 0) return GSN_ERR_INVALID_ARGUMENT;
    std::vector<gs_native::CameraParams> cams;
    std::vector<const uint8_t*> imgs;
    for (int k = 0; k < count; ++k) {
        cams.push_back(AsCamera(cameras + k));
        imgs.push_back(images[k]);
    }
    return t->impl.EvaluateMetrics(cams, imgs, psnr, ssim, l1, loss) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_spatial_permutation(const float* params, int count, uint32_t* perm, void* stream) {
    if (!params || !perm || count <= 0) return GSN_ERR_INVALID_ARGUMENT;
    gs_native::SpatialOrder order;
    order.SetStream(static_cast<cudaStream_t>(stream));
    if (!order.Compute(params, count)) return GSN_ERR_CUDA;
    if (cudaMemcpyAsync(perm, order.GetPermutation(), sizeof(uint32_t) * count, cudaMemcpyDeviceToDevice,
                        static_cast<cudaStream_t>(stream)) != cudaSuccess ||
        cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess)
        return GSN_ERR_CUDA;
    return GSN_OK;
}

int gsn_gather_gaussians(const float* src, float* dst, const uint32_t* perm, int count, int bf16_sh, void* stream) {
    if (!src || !dst || !perm || count <= 0 || src == dst) return GSN_ERR_INVALID_ARGUMENT;
    return gsn::launch_gather_gaussians(src, dst, perm, count, bf16_sh != 0, static_cast<cudaStream_t>(stream));
}

int gsn_eval_metrics(const float* image, const uint8_t* target, int width, int height, double* out, void* stream) {
    if (!image || !target || !out || width <= 0 || height <= 0) return GSN_ERR_INVALID_ARGUMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    gs_native::DeviceArray<double> workspace, metrics;
    if (!workspace.Reserve(gsn::eval_metrics_workspace(width, height) / sizeof(double)) || !metrics.Reserve(4))
        return GSN_ERR_OUT_OF_MEMORY;
    const int st = gsn::launch_eval_metrics(image, target, width, height, workspace.get(), metrics.get(), s);
    if (st != GSN_OK) return st;
    if (cudaMemcpyAsync(out, metrics.get(), 4 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GSN_ERR_CUDA;
    return GSN_OK;
}

int gsn_trainer_save(gsn_trainer* t, const char* path) {
    if (!t || !path) return GSN_ERR_INVALID_ARGUMENT;
    return t->impl.Save(path) ? GSN_OK : GSN_ERR_IO;
}

int gsn_trainer_load(gsn_trainer* t, const char* path) {
    if (!t || !path) return GSN_ERR_INVALID_ARGUMENT;
    return t->impl.Load(path) ? GSN_OK : GSN_ERR_IO;
}

int gsn_trainer_state(gsn_trainer* t, float** params, int* count, int* completed, int* sh_degree,
                      float* scene_extent) {
    if (!t) return GSN_ERR_INVALID_ARGUMENT;
    if (params) *params = t->impl.GetGaussians().gaussians_;
    if (count) *count = t->impl.GetGaussians().gaussian_count_;
    if (completed) *completed = t->impl.GetCompleted();
    if (sh_degree) *sh_degree = t->impl.GetShDegree();
    if (scene_extent) *scene_extent = t->impl.GetSceneExtent();
    return GSN_OK;
}

int gsn_ply_write(const char* path, const float* params, int count) {
    if (!path || count < 0 || (count > 0 && !params)) return GSN_ERR_INVALID_ARGUMENT;
    return gs_native::WriteGaussiansPly(path, gs_native::UnpackGaussians(params, count)) ? GSN_OK : GSN_ERR_IO;
}

int gsn_ply_read_count(const char* path, int* count) {
    if (!path || !count) return GSN_ERR_INVALID_ARGUMENT;
    std::vector<gs_native::Gaussian> g;
    if (!gs_native::ReadGaussiansPly(path, g)) return GSN_ERR_IO;
    *count = static_cast<int>(g.size());
    return GSN_OK;
}

int gsn_ply_read(const char* path, float* params, int count) {
    if (!path || !params || count <= 0) return GSN_ERR_INVALID_ARGUMENT;
    std::vector<gs_native::Gaussian> g;
    if (!gs_native::ReadGaussiansPly(path, g)) return GSN_ERR_IO;
    if (static_cast<int>(g.size()) != count) return GSN_ERR_INVALID_ARGUMENT;
    std::vector<float> p = gs_native::PackGaussians(g);
    std::copy(p.begin(), p.end(), params);
    return GSN_OK;
}

// ---------------------------------------------------------------- batched form
int gsn_graph_create(gsn_graph** out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    *out = new (std::nothrow) gsn_graph();
    return *out ? GSN_OK : GSN_ERR_OUT_OF_MEMORY;
}

int gsn_graph_destroy(gsn_graph* g) {
    delete g;
    return GSN_OK;
}

int gsn_graph_capture(gsn_graph* g, gsn_renderer* renderer, gsn_solver* solver, float* params, int count,
                      const gsn_camera* cameras, int camera_count, const uint8_t* device_targets,
                      size_t target_stride, const float* background, float* device_image, int sh_degree,
                      int64_t record_capacity, void* stream) {
    if (!g || !renderer || !solver || !params || count <= 0 || !cameras || camera_count <= 0 || !background)
        return GSN_ERR_INVALID_ARGUMENT;
    std::vector<gs_native::CameraParams> cams(static_cast<size_t>(camera_count));
    for (int k = 0; k < camera_count; ++k) cams[k] = AsCamera(cameras + k);
    g->gaussians = View(params, count);
    return g->impl.Capture(renderer->impl, solver->impl, g->gaussians, cams, device_targets, target_stride,
                           background, device_image, sh_degree, record_capacity, AsStream(stream))
               ? GSN_OK
               : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_graph_run(gsn_graph* g, const int* views, const float* position_lrs, int steps) {
    if (!g) return GSN_ERR_INVALID_ARGUMENT;
    if (!g->impl.Captured()) return GSN_ERR_NOT_READY;
    return g->impl.Run(views, position_lrs, steps) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_graph_check(gsn_graph* g) {
    if (!g) return GSN_ERR_INVALID_ARGUMENT;
    return g->impl.Check();
}

int gsn_graph_launches_per_step(gsn_graph* g, int* out) {
    if (!g || !out) return GSN_ERR_INVALID_ARGUMENT;
    *out = g->impl.LaunchesPerStep();
    return GSN_OK;
}

// ---------------------------------------------------------------- tensor cores
int gsn_tc_gemm_selftest(const float* a, const float* b, float* d, void* stream) {
    int* status = nullptr;
    if (cudaMalloc(&status, sizeof(int)) != cudaSuccess) return GSN_ERR_OUT_OF_MEMORY;
    int result = cudaMemsetAsync(status, 0, sizeof(int), AsStream(stream)) == cudaSuccess ? GSN_OK : GSN_ERR_CUDA;
    if (result == GSN_OK) result = gsn::launch_tc_gemm_selftest(a, b, d, status, AsStream(stream));
    int host_status = GSN_OK;
    if (result == GSN_OK &&
        (cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, AsStream(stream)) != cudaSuccess ||
         cudaStreamSynchronize(AsStream(stream)) != cudaSuccess))
        result = GSN_ERR_CUDA;
    cudaFree(status);
    return result == GSN_OK ? host_status : result;
}

// ---------------------------------------------------------------- learned density
int gsn_trainer_save_checkpoint(gsn_trainer* t, const char* path) {
    if (!t || !path) return GSN_ERR_INVALID_ARGUMENT;
    return t->impl.SaveCheckpoint(path) ? GSN_OK : GSN_ERR_IO;
}

int gsn_trainer_load_checkpoint(gsn_trainer* t, const char* path) {
    if (!t || !path) return GSN_ERR_INVALID_ARGUMENT;
    return t->impl.LoadCheckpoint(path) ? GSN_OK : GSN_ERR_IO;
}

int gsn_trainer_set_density_mlp(gsn_trainer* t, const float* weights) {
    if (!t || !weights) return GSN_ERR_INVALID_ARGUMENT;
    return t->impl.SetDensityMlp(weights) ? GSN_OK : GSN_ERR_CUDA;
}

int gsn_trainer_density_log(gsn_trainer* t, const float** features, const int8_t** decisions, const int** parents,
                            int* before, int* after, int* steps, int* iteration) {
    if (!t) return GSN_ERR_INVALID_ARGUMENT;
    const gs_native::DensityLog& log = t->impl.GetDensityLog();
    if (features) *features = log.features;
    if (decisions) *decisions = log.decisions;
    if (parents) *parents = log.parents;
    if (before) *before = log.before;
    if (after) *after = log.after;
    if (steps) *steps = log.steps;
    if (iteration) *iteration = log.iteration;
    return GSN_OK;
}

int gsn_mlp_create(gsn_mlp** out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    *out = new (std::nothrow) gsn_mlp();
    return *out ? GSN_OK : GSN_ERR_OUT_OF_MEMORY;
}

int gsn_mlp_destroy(gsn_mlp* m) {
    delete m;
    return GSN_OK;
}

int gsn_mlp_initialize(gsn_mlp* m, unsigned long long seed) {
    if (!m) return GSN_ERR_INVALID_ARGUMENT;
    return m->impl.Initialize(seed) ? GSN_OK : GSN_ERR_CUDA;
}

int gsn_mlp_set_weights(gsn_mlp* m, const float* host_weights) {
    if (!m || !host_weights) return GSN_ERR_INVALID_ARGUMENT;
    return m->impl.SetWeights(host_weights) ? GSN_OK : GSN_ERR_CUDA;
}

int gsn_mlp_get_weights(gsn_mlp* m, float* host_weights) {
    if (!m || !host_weights) return GSN_ERR_INVALID_ARGUMENT;
    return m->impl.GetWeights(host_weights) ? GSN_OK : GSN_ERR_NOT_READY;
}

int gsn_mlp_gradients(gsn_mlp* m, const float* features, const int* labels, const float* weights, int n,
                      float* host_grad, double* loss) {
    if (!m) return GSN_ERR_INVALID_ARGUMENT;
    return m->impl.Gradients(features, labels, weights, n, host_grad, loss) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_mlp_train(gsn_mlp* m, const float* features, const int* labels, const float* weights, int n, int steps,
                  float lr, double* loss) {
    if (!m) return GSN_ERR_INVALID_ARGUMENT;
    return m->impl.Train(features, labels, weights, n, steps, lr, loss) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_mlp_infer(gsn_mlp* m, const float* features, int n, float confidence, int8_t* actions, float* probs) {
    if (!m) return GSN_ERR_INVALID_ARGUMENT;
    return m->impl.Infer(features, n, confidence, actions, probs) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

// ---------------------------------------------------------------- multi-view renderer
int gsn_multiview_create(gsn_multiview** out) {
    if (!out) return GSN_ERR_INVALID_ARGUMENT;
    *out = new (std::nothrow) gsn_multiview();
    return *out ? GSN_OK : GSN_ERR_OUT_OF_MEMORY;
}

int gsn_multiview_destroy(gsn_multiview* m) {
    delete m;
    return GSN_OK;
}

int gsn_multiview_set_stream(gsn_multiview* m, void* stream) {
    if (!m) return GSN_ERR_INVALID_ARGUMENT;
    m->impl.SetStream(AsStream(stream));
    return GSN_OK;
}

int gsn_multiview_set_config(gsn_multiview* m, int tile_w, int tile_h, int threads, int key_bits) {
    if (!m) return GSN_ERR_INVALID_ARGUMENT;
    return m->impl.SetConfig({tile_w, tile_h, threads, key_bits}) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_multiview_get_config(gsn_multiview* m, int* tile_w, int* tile_h, int* threads, int* key_bits) {
    if (!m || !tile_w || !tile_h || !threads || !key_bits) return GSN_ERR_INVALID_ARGUMENT;
    const gs_native::MultiViewConfig& c = m->impl.GetConfig();
    *tile_w = c.tile_w;
    *tile_h = c.tile_h;
    *threads = c.threads;
    *key_bits = c.key_bits;
    return GSN_OK;
}

namespace {

bool MultiViewInputs(const gsn_camera* cameras, int views, float* const* images,
                     std::vector<gs_native::CameraParams>& cams, std::vector<float*>& imgs) {
    if (!cameras || !images || views <= 0) return false;
    cams.resize(static_cast<size_t>(views));
    imgs.resize(static_cast<size_t>(views));
    for (int k = 0; k < views; ++k) {
        cams[k] = AsCamera(cameras + k);
        imgs[k] = images[k];
    }
    return true;
}

}  // namespace

int gsn_multiview_render(gsn_multiview* m, const float* params, int count, const gsn_camera* cameras, int views,
                         float* const* images, const float* background, int sh_degree) {
    std::vector<gs_native::CameraParams> cams;
    std::vector<float*> imgs;
    if (!m || !background || !MultiViewInputs(cameras, views, images, cams, imgs)) return GSN_ERR_INVALID_ARGUMENT;
    return m->impl.Render(View(params, count), cams, background, imgs, sh_degree) ? GSN_OK
                                                                                   : GSN_ERR_INVALID_ARGUMENT;
}

int gsn_multiview_autotune(gsn_multiview* m, const float* params, int count, const gsn_camera* cameras, int views,
                           float* const* images, const float* background, int sh_degree, int repeats,
                           float* results, int max_results, int* result_count) {
    std::vector<gs_native::CameraParams> cams;
    std::vector<float*> imgs;
    if (!m || !background || !MultiViewInputs(cameras, views, images, cams, imgs)) return GSN_ERR_INVALID_ARGUMENT;
    std::vector<gs_native::MultiViewTiming> timings;
    if (!m->impl.Autotune(View(params, count), cams, background, imgs, sh_degree, repeats, &timings))
        return GSN_ERR_CUDA;
    const int rows = std::min(static_cast<int>(timings.size()), std::max(max_results, 0));
    for (int k = 0; results && k < rows; ++k) {
        const gs_native::MultiViewTiming& t = timings[k];
        results[5 * k + 0] = static_cast<float>(t.config.tile_w);
        results[5 * k + 1] = static_cast<float>(t.config.tile_h);
        results[5 * k + 2] = static_cast<float>(t.config.threads);
        results[5 * k + 3] = static_cast<float>(t.config.key_bits);
        results[5 * k + 4] = static_cast<float>(t.ms);
    }
    if (result_count) *result_count = static_cast<int>(timings.size());
    return GSN_OK;
}

struct gsn_scene {
    gs_native::ColmapScene impl;
};

int gsn_scene_read_colmap(const char* scene_dir, int downscale, gsn_scene** out) {
    if (!scene_dir || !out) return GSN_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    gsn_scene* s = new (std::nothrow) gsn_scene;
    if (!s) return GSN_ERR_OUT_OF_MEMORY;
    if (!gs_native::ReadColmapScene(scene_dir, downscale, s->impl)) {
        delete s;
        return GSN_ERR_IO;
    }
    *out = s;
    return GSN_OK;
}

int gsn_scene_destroy(gsn_scene* s) {
    delete s;
    return GSN_OK;
}

int gsn_scene_counts(const gsn_scene* s, int* train, int* test, int* points) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    if (train) *train = static_cast<int>(s->impl.train_cameras.size());
    if (test) *test = static_cast<int>(s->impl.test_cameras.size());
    if (points) *points = static_cast<int>(s->impl.point_positions.size() / 3);
    return GSN_OK;
}

int gsn_scene_view(const gsn_scene* s, int split, int index, gsn_camera* camera, const uint8_t** image,
                   const char** name) {
    if (!s || (split != 0 && split != 1)) return GSN_ERR_INVALID_ARGUMENT;
    const auto& cams = split == 0 ? s->impl.train_cameras : s->impl.test_cameras;
    const auto& imgs = split == 0 ? s->impl.train_images : s->impl.test_images;
    const auto& names = split == 0 ? s->impl.train_names : s->impl.test_names;
    if (index < 0 || index >= static_cast<int>(cams.size())) return GSN_ERR_INVALID_ARGUMENT;
    if (camera) *camera = gs_native::AsGsnCamera(cams[index]);
    if (image) *image = imgs[index].rgb.data();
    if (name) *name = names[index].c_str();
    return GSN_OK;
}

int gsn_scene_points(const gsn_scene* s, const float** positions, const float** colors) {
    if (!s) return GSN_ERR_INVALID_ARGUMENT;
    if (positions) *positions = s->impl.point_positions.data();
    if (colors) *colors = s->impl.point_colors.data();
    return GSN_OK;
}

static bool AsImage(const uint8_t* rgb, int width, int height, gs_native::ImageU8& image) {
    if (!rgb || width <= 0 || height <= 0) return false;
    image.width = width;
    image.height = height;
    image.rgb.assign(rgb, rgb + static_cast<size_t>(width) * height * 3);
    return true;
}

int gsn_image_write_ppm(const char* path, const uint8_t* rgb, int width, int height) {
    gs_native::ImageU8 image;
    if (!path || !AsImage(rgb, width, height, image)) return GSN_ERR_INVALID_ARGUMENT;
    return gs_native::WritePpm(path, image) ? GSN_OK : GSN_ERR_IO;
}

int gsn_image_write_png(const char* path, const uint8_t* rgb, int width, int height) {
    gs_native::ImageU8 image;
    if (!path || !AsImage(rgb, width, height, image)) return GSN_ERR_INVALID_ARGUMENT;
    return gs_native::WritePng(path, image) ? GSN_OK : GSN_ERR_IO;
}

}  // extern "C"
