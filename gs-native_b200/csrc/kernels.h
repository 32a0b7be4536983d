// Internal launcher interface of the gs-native B200 kernels. Host C++ code (the
// C ABI in abi.cpp and the drop-in classes) calls these; every launcher is
// asynchronous on the given stream and returns a gsn status code.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "gsn_types.h"

namespace gsn {

// ---------------------------------------------------------------- projection
struct ProjectOutputs {
    float2* means;           // [N] pixel-space centre (u, v)
    float4* conic_opacity;   // [N] inverse 2D covariance (a, b, c) + sigmoid opacity
    float3* colors;          // [N] SH colour, clamped below at 0
    float* depths;           // [N] camera-space z
    int4* rects;             // [N] tile rectangle [x0, y0, x1, y1)
    int* tile_counts;        // [N] tiles touched (0 = culled)
    uint32_t* depth_keys;    // [N] float bits of z, 0xFFFFFFFF when culled
    float* radii;            // [N] optional 3-sigma pixel radius (0 = culled), may be null
};
int launch_project(const float* params, int n, const gsn_camera& cam, int sh_degree,
                   const ProjectOutputs& out, cudaStream_t stream);

// ---------------------------------------------------------------- sorting
// Stable LSD radix sort of (uint32 key, uint32 value) pairs over key bits
// [begin_bit, end_bit). Ping-pongs between (keys, values) and (keys_alt,
// values_alt); on return *result_in_alt tells which pair holds the sorted
// output. With identity_values the first pass reads the values 0..n-1 instead of
// `values`. `count` may live on the device (count_device != null): the launch
// grid is sized for `max_count` and every kernel reads the actual count from
// device memory, so no host sync is needed.
struct RadixSortScratch {
    uint32_t* block_hist;   // [256 * max_blocks]
    uint32_t* digit_total;  // [256 * passes]
    size_t max_blocks;
};
size_t radix_sort_scratch_bytes(int max_count);
RadixSortScratch radix_sort_scratch(void* base, int max_count);
int launch_radix_sort(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt,
                      bool identity_values, int max_count, const int* count_device, int begin_bit,
                      int end_bit, const RadixSortScratch& scratch, bool* result_in_alt,
                      cudaStream_t stream);

// Exclusive prefix sum of 32-bit integers, in -> out (in-place allowed), n + 1
// outputs with out[n] = total. `gather` (optional) reads in[gather[i]] instead of
// in[i]. Scratch: scan_scratch_bytes(n).
size_t scan_scratch_bytes(int n);
int launch_exclusive_scan(const int* in, const uint32_t* gather, int* out, int n, void* scratch,
                          cudaStream_t stream);

// Emit one (tile, gaussian id) record per tile of every visible Gaussian, in
// depth order. record_start[p] is the exclusive scan of tile counts in sorted
// order; records beyond `capacity` are not written and set *overflow.
int launch_emit_records(const uint32_t* sorted_ids, const int* record_start, const int4* rects,
                        int n, int tile_count_x, uint32_t* tile_keys, uint32_t* record_ids,
                        int64_t capacity, int* overflow, cudaStream_t stream);

// Per-tile [begin, end) offsets of sorted tile keys (empty tiles included).
int launch_tile_ranges(const uint32_t* sorted_tiles, const int* record_count_device, int max_records,
                       int tile_count, int64_t* offsets, cudaStream_t stream);

// ---------------------------------------------------------------- raster
struct RasterForwardArgs {
    const uint32_t* tile_ids;      // sorted Gaussian id per record
    const int64_t* tile_offsets;   // [T + 1]
    const float2* means;
    const float4* conic_opacity;
    const float3* colors;
    gsn_camera cam;
    float3 background;
    float* image;                  // HWC RGB fp32
    float* final_transmittance;    // [P] optional
    int* contributors;             // [P] optional: records consumed before the pixel finished
};
int launch_raster_forward(const RasterForwardArgs& a, cudaStream_t stream);

}  // namespace gsn
