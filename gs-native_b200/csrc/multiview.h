// Launchers of the multi-view renderer (multiview.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gsn {

// Per-view inputs of the persistent blend (device pointers).
struct MultiView {
    const uint32_t* tile_ids;     // sorted record ids
    const int64_t* tile_offsets;  // [tiles + 1]
    const float2* means;
    const float4* conic_opacity;
    const float3* colors;
    float* image;                 // fp32 HWC
    int width, height, tiles_x, tiles_y;
    float3 background;
};

struct MultiViewArgs {
    const MultiView* views;   // [view_count] (device)
    const int* tile_prefix;   // [view_count + 1] exclusive prefix of tile counts (device)
    int* queue;               // work counter, zero before the launch
    int view_count;
    int total_tiles;
};

// Tile shapes 16x16, 16x8, 8x8 with 64, 128 or 256 threads where every thread
// owns at least one pixel row of its warp's strip.
bool multiview_config_valid(int tile_w, int tile_h, int threads);
int launch_multiview(const MultiViewArgs& a, int tile_w, int tile_h, int threads, cudaStream_t stream);
// Records of every visible Gaussian in id order with its depth key (48/64-bit orders).
int launch_emit_keyed(const int* record_start, const int4* rects, const int* tile_counts, const uint32_t* depth_bits,
                      int n, int tiles_x, int64_t capacity, uint32_t* tile_keys, uint32_t* depth_keys, uint32_t* ids,
                      cudaStream_t stream);
// tiles_out[p] = tile_keys[order[p]], ids_out[p] = ids[order[p]].
int launch_gather_records(const uint32_t* order, const uint32_t* tile_keys, const uint32_t* ids, int64_t count,
                          uint32_t* tiles_out, uint32_t* ids_out, cudaStream_t stream);

}  // namespace gsn
