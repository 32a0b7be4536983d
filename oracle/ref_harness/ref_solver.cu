// Test-infrastructure harness: the reference's solver (src/core/solver/solver.cu,
// compiled unmodified from the reference tree) behind extern "C" entry points,
// both the Solver class and its individual kernels. Not part of the product.
#include "core/solver/solver.cu"

using gs_native::CameraParams;
using gs_native::GaussianBuffers;
using gs_native::Renderer;
using gs_native::Solver;

extern "C" {

int ref_solver_create(void** out) {
    *out = new Solver();
    return 0;
}

int ref_solver_destroy(void* h) {
    delete static_cast<Solver*>(h);
    return 0;
}

// Solver::Iterate (solver.cu:702-720).
int ref_solver_iterate(void* h, const CameraParams* cam, void* renderer, const float* image, const uint8_t* target,
                       float* params, int count, float position_lr, int sh_degree) {
    GaussianBuffers g;
    g.gaussians_ = params;
    g.gaussian_count_ = count;
    bool ok = static_cast<Solver*>(h)->Iterate(*cam, *static_cast<Renderer*>(renderer), image, target, g,
                                               position_lr, sh_degree);
    return ok && cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

int ref_solver_reset_opacity_history(void* h) { return static_cast<Solver*>(h)->ResetOpacityHistory() ? 0 : -1; }

int ref_solver_remap(void* h, const int* parent_ids, int count) {
    return static_cast<Solver*>(h)->RemapGaussians(parent_ids, count) ? 0 : -1;
}

int ref_solver_stats(void* h, const float** stats, const float** abs_stats) {
    *stats = static_cast<Solver*>(h)->GetProjectionStatistics();
    *abs_stats = static_cast<Solver*>(h)->GetAbsoluteProjectionStatistics();
    return 0;
}

// ComputeImageGradientsKernel (solver.cu:26-168), launched as solver.cu:752-757.
int ref_image_gradients(const float* image, const uint8_t* target, float* gradients, int width, int height) {
    dim3 grid((width + 15) / 16, (height + 31) / 32, 3);
    gs_native::ComputeImageGradientsKernel<<<grid, 512>>>(image, target, gradients, width, height);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// ComputeSplatGradientsKernel (solver.cu:325-466) into a zeroed 58 x count
// gradient block and a zeroed 2 x count absolute block (rows 0-8 / 0-1 written).
int ref_splat_gradients(const int* ids, const int64_t* offsets, const float2* means, const float4* conic,
                        const float3* colors, const float* image, const float* image_gradients,
                        const CameraParams* cam, float* gradients, float* absolute, int count) {
    int tiles = cam->tile_count_x_ * cam->tile_count_y_;
    gs_native::ComputeSplatGradientsKernel<<<tiles, 256>>>(ids, offsets, means, conic, colors, image,
                                                           image_gradients, *cam, gradients, absolute, count);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// CollectProjectionStatisticsKernel (solver.cu:468-490).
int ref_projection_statistics(const float* gradients, const int* record_offsets, float* statistics,
                              float* absolute, int count, int width, int height) {
    gs_native::CollectProjectionStatisticsKernel<<<(count + 255) / 256, 256>>>(
        gradients, record_offsets, statistics, absolute, count, width, height);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// MapGaussianGradientsKernel<D> (solver.cu:492-623), in place on rows 0-57.
int ref_map_gradients(const float* params, const CameraParams* cam, float* gradients, int count, int sh_degree) {
    int grid = (count + 255) / 256;
    switch (sh_degree) {
        case 0: gs_native::MapGaussianGradientsKernel<0><<<grid, 256>>>(params, *cam, gradients, count); break;
        case 1: gs_native::MapGaussianGradientsKernel<1><<<grid, 256>>>(params, *cam, gradients, count); break;
        case 2: gs_native::MapGaussianGradientsKernel<2><<<grid, 256>>>(params, *cam, gradients, count); break;
        default: gs_native::MapGaussianGradientsKernel<3><<<grid, 256>>>(params, *cam, gradients, count); break;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// UpdateGaussiansKernel (solver.cu:651-689) with the host bias corrections of
// solver.cu:912-914 for step `iteration` (1-based).
int ref_adam(const float* gradients, float* params, float* first, float* second, int count, float position_lr,
             unsigned long long iteration) {
    float c1 = static_cast<float>(1.0 / (1.0 - std::pow(0.9, static_cast<double>(iteration))));
    float c2 = static_cast<float>(1.0 / (1.0 - std::pow(0.999, static_cast<double>(iteration))));
    dim3 grid((count + 255) / 256, gs_native::kMaxParamCount);
    gs_native::UpdateGaussiansKernel<<<grid, 256>>>(gradients, params, first, second, count, position_lr, c1, c2);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// The steady-state loop of GaussianSplatting::Train (gaussian_splatting.cpp:
// 137-187, iterations >= 15000: no density statistics, no density control, no
// opacity reset; the per-iteration log line is not emitted) over the
// reference's own Renderer and Solver: per step the view's target is uploaded
// from host memory with cudaMemcpy2D as Train does (host_targets != nullptr) or
// read from device memory (device_targets), then Render and Iterate. views[k]
// is step k's camera index into cameras / the targets (width * height * 3
// bytes each). The loop's device time (CUDA events on the legacy stream the
// reference uses) is written to elapsed_ms. Timing harness only.
int ref_train_replay(void* renderer, void* solver, float* params, int count, const CameraParams* cameras,
                     const int* views, int steps, const uint8_t* const* host_targets, const uint8_t* device_targets,
                     uint8_t* target_buffer, const float* background, float* image, float position_lr,
                     int sh_degree, float* elapsed_ms) {
    auto* r = static_cast<Renderer*>(renderer);
    auto* s = static_cast<Solver*>(solver);
    GaussianBuffers g;
    g.gaussians_ = params;
    g.gaussian_count_ = count;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -1;
    int status = 0;
    cudaEventRecord(e0, 0);
    for (int k = 0; k < steps && status == 0; ++k) {
        const CameraParams& cam = cameras[views[k]];
        const size_t row = static_cast<size_t>(cam.width_) * 3;
        const uint8_t* target = nullptr;
        if (host_targets) {
            if (cudaMemcpy2D(target_buffer, row, host_targets[views[k]], row, row, cam.height_,
                             cudaMemcpyHostToDevice) != cudaSuccess)
                status = -2;
            target = target_buffer;
        } else {
            target = device_targets + static_cast<size_t>(views[k]) * row * cam.height_;
        }
        if (status == 0 && !r->Render(g, cam, background, image, sh_degree)) status = -3;
        if (status == 0 && !s->Iterate(cam, *r, image, target, g, position_lr, sh_degree)) status = -4;
    }
    cudaEventRecord(e1, 0);
    if (cudaEventSynchronize(e1) != cudaSuccess) status = status ? status : -5;
    cudaEventElapsedTime(elapsed_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return status;
}

}  // extern "C"
