// Test-infrastructure harness: exposes the reference's own renderer
// (src/core/render/renderer.cu, compiled unmodified from the reference tree by
// oracle/Makefile) through extern "C" so the parity tests can run it beside the
// gs-native kernels on identical device inputs. Not part of the product.
#include "core/render/renderer.cu"

using gs_native::CameraParams;
using gs_native::GaussianBuffers;
using gs_native::Renderer;

extern "C" {

int ref_renderer_create(void** out) {
    *out = new Renderer();
    return 0;
}

int ref_renderer_destroy(void* h) {
    delete static_cast<Renderer*>(h);
    return 0;
}

// Renderer::Render (renderer.cu:359-372).
int ref_renderer_render(void* h, const float* params, int count, const CameraParams* cam, const float* bg,
                        float* image, int sh_degree) {
    GaussianBuffers g;
    g.gaussians_ = const_cast<float*>(params);
    g.gaussian_count_ = count;
    return static_cast<Renderer*>(h)->Render(g, *cam, bg, image, sh_degree) ? 0 : -1;
}

// Public getters of renderer.h:28-54.
int ref_renderer_get(void* h, const void** means, const void** conic, const void** colors, const int** tile_ids,
                     const int64_t** tile_offsets, const int** record_offsets, int* gaussian_capacity,
                     int* tile_capacity) {
    auto* r = static_cast<Renderer*>(h);
    *means = r->GetMeans();
    *conic = r->GetConicOpacities();
    *colors = r->GetColors();
    *tile_ids = r->GetTileGaussianIds();
    *tile_offsets = r->GetTileGaussianOffsets();
    *record_offsets = r->GetRecordOffsets();
    *gaussian_capacity = r->GetGaussianCapacity();
    *tile_capacity = r->GetTileCapacity();
    return 0;
}

// ProjectGaussiansKernel (renderer.cu:108-221) into caller buffers, so the
// depth and tile-rect outputs private to the class can be compared too.
int ref_project(const float* params, int count, const CameraParams* cam, int sh_degree, float2* means,
                float4* conic, float3* colors, float* depths, int4* rects, int* record_offsets) {
    if (count <= 0) return 0;
    gs_native::ProjectGaussiansKernel<<<(count + 255) / 256, 256>>>(params, *cam, means, conic, colors, depths,
                                                                   rects, record_offsets, count, sh_degree);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

}  // extern "C"
