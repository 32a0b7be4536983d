// Test-infrastructure harness: the reference's density controller
// (src/core/density/density_controller.cu, compiled unmodified from the
// reference tree) behind extern "C". Not part of the product.
#include "core/density/density_controller.cu"

using gs_native::DensityController;
using gs_native::GaussianBuffers;

extern "C" {

int ref_density_create(void** out) {
    *out = new DensityController();
    return 0;
}

int ref_density_destroy(void* h) {
    delete static_cast<DensityController*>(h);
    return 0;
}

int ref_density_initialize(void* h, int count, int capacity) {
    return static_cast<DensityController*>(h)->Initialize(count, capacity) ? 0 : -1;
}

int ref_density_accumulate_observations(void* h, const float* gradients, const float* radii, const int* ids,
                                        int observations) {
    return static_cast<DensityController*>(h)->AccumulateStatistics(gradients, radii, ids, observations) ? 0 : -1;
}

int ref_density_accumulate(void* h, const float* statistics, const float* absolute, int count) {
    return static_cast<DensityController*>(h)->AccumulateStatistics(statistics, absolute, count) ? 0 : -1;
}

int ref_density_reset_opacity(void* h, float* params, int stride, float max_opacity) {
    return static_cast<DensityController*>(h)->ResetOpacity(params, stride, max_opacity) ? 0 : -1;
}

// DensityController::ControlDensity (density_controller.cu:461-611). On success
// *params / *count receive the swapped-in buffer (ownership ping-pong).
int ref_density_control(void* h, float** params, int* count, float scene_extent, float gradient_threshold,
                        float percent_dense, float min_opacity, float max_screen_size, unsigned long long seed,
                        int* changes, float absolute_gradient_threshold) {
    GaussianBuffers g;
    g.gaussians_ = *params;
    g.gaussian_count_ = *count;
    bool ok = static_cast<DensityController*>(h)->ControlDensity(g, scene_extent, gradient_threshold, percent_dense,
                                                                 min_opacity, max_screen_size, seed, changes,
                                                                 absolute_gradient_threshold);
    *params = g.gaussians_;
    *count = g.gaussian_count_;
    return ok && cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

int ref_density_get(void* h, const int** history_parents, const int** control, const int** parents) {
    auto* d = static_cast<DensityController*>(h);
    *history_parents = d->GetHistoryParentIds();
    *control = d->GetGaussianCount();
    *parents = d->GetParentIds();
    return 0;
}

}  // extern "C"
