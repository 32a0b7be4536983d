// extern "C" ABI of the gs-native B200 library (declarations in include/gsn.h).
#include "gsn.h"

#include <cuda_runtime.h>

#include <new>

#include "core/render/renderer.h"

struct gsn_renderer {
    gs_native::Renderer impl;
};

namespace {

inline cudaStream_t AsStream(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

const char* gsn_version(void) { return "gs-native-b200 0.1.0 (sm_100a)"; }

int gsn_memcpy(void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return GSN_OK;
    if (!dst || !src) return GSN_ERR_INVALID_ARGUMENT;
    return cudaMemcpy(dst, src, bytes, cudaMemcpyDefault) == cudaSuccess ? GSN_OK : GSN_ERR_CUDA;
}

int gsn_stream_synchronize(void* stream) {
    return cudaStreamSynchronize(AsStream(stream)) == cudaSuccess ? GSN_OK : GSN_ERR_CUDA;
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

int gsn_renderer_set_record_capacity(gsn_renderer* r, int64_t records) {
    if (!r) return GSN_ERR_INVALID_ARGUMENT;
    return r->impl.SetRecordCapacity(records) ? GSN_OK : GSN_ERR_INVALID_ARGUMENT;
}

}  // extern "C"
