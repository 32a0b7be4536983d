// Multi-view forward renderer (gs-native extension; the reference renders one
// view per call, renderer.cu:359-590): any number of views of uneven
// resolution rendered with one persistent blend launch over all of their
// tiles, plus an autotuner over tile shape, threads per tile and sort key
// width.
//
// Per view the preprocessing is the single-view renderer's (projection, record
// ordering, per-tile ranges) into buffers of its own, the views spread over
// eight side streams so their small launches overlap; all views' record totals
// are read back with one synchronisation, and one persistent kernel then blends
// every (view, tile) work item. Sort key width: 32 = a stable sort of the N
// depth keys, records emitted in depth order, then a stable sort on the tile
// bits only; 48 = records emitted in id order, stable sort on the 32 depth
// bits then on the ceil(log2 tiles) tile bits (the reference's 32 + log2 T
// bits); 64 = the same with all 32 tile bits. All three give the same per-tile
// order (tile, depth, id).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "core/types/buffers.h"
#include "util/device_array.h"

namespace gs_native {

struct MultiViewConfig {
    int tile_w = 16;
    int tile_h = 16;
    int threads = 64;
    int key_bits = 32;
};

struct MultiViewTiming {
    MultiViewConfig config;
    double ms = 0.0;  // device time of one multi-view render (mean over repeats)
};

class MultiViewRenderer {
public:
    MultiViewRenderer();
    ~MultiViewRenderer();
    MultiViewRenderer(const MultiViewRenderer&) = delete;
    MultiViewRenderer& operator=(const MultiViewRenderer&) = delete;

    void SetStream(cudaStream_t stream) { stream_ = stream; }
    bool SetConfig(const MultiViewConfig& config);
    const MultiViewConfig& GetConfig() const { return config_; }
    static bool ConfigValid(const MultiViewConfig& config);

    // Renders cameras[v] into device fp32 HWC images[v] (width * height * 3).
    // Camera tile counts are recomputed for the configured tile shape.
    bool Render(const GaussianBuffers& gaussians, const std::vector<CameraParams>& cameras,
                const float background[3], const std::vector<float*>& images, int sh_degree);
    // Times every valid configuration (repeats renders each) on these views,
    // keeps the fastest and returns all timings.
    bool Autotune(const GaussianBuffers& gaussians, const std::vector<CameraParams>& cameras,
                  const float background[3], const std::vector<float*>& images, int sh_degree, int repeats,
                  std::vector<MultiViewTiming>* timings);
    int64_t GetLastRecordCount() const { return last_records_; }

private:
    struct View;
    bool Prepare(View& v, const GaussianBuffers& g, const CameraParams& cam, int sh_degree, cudaStream_t stream);
    bool Order(View& v, int count, cudaStream_t stream);
    bool EnsureSideStreams();

    // The views' projection and record ordering (small, latency-bound
    // launches) run concurrently on kSideStreams streams of the renderer's
    // own; the persistent blend runs on the caller's stream after all of them.
    static constexpr int kSideStreams = 8;
    std::vector<cudaStream_t> side_;
    std::vector<cudaEvent_t> joins_;
    cudaEvent_t fork_ = nullptr;
    cudaStream_t stream_ = nullptr;
    MultiViewConfig config_;
    std::vector<std::unique_ptr<View>> views_;
    DeviceArray<unsigned char> table_;  // MultiView[views] + tile prefix + queue
    int* host_totals_ = nullptr;       // pinned, one per view
    size_t host_totals_count_ = 0;
    int64_t last_records_ = 0;
};

}  // namespace gs_native
