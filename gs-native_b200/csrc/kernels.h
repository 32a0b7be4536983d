// Internal launcher interface of the gs-native B200 kernels. Host C++ code (the
// C ABI in abi.cpp and the drop-in classes) calls these; every launcher is
// asynchronous on the given stream and returns a gsn status code.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "gsn_types.h"

namespace gsn {

// ---------------------------------------------------------------- step frame
// Per-iteration values that the batched (CUDA graph) form keeps in device
// memory, so that one captured iteration serves every step: the view's camera,
// its resident training target and the step's scalars. Kernels given a frame
// read these instead of their by-value arguments. All views of one graph share
// the resolution (and so the tile grid and record layout) it was captured with.
struct StepFrame {
    gsn_camera cam;
    const uint8_t* target;
    float position_lr;
    float c1, c2;  // Adam bias corrections of this step
    uint32_t seed; // stochastic-rounding seed of this step (precision form)
    int view;
    int step;      // index into the schedule
};

// Host-written schedule read by the frame kernel at the start of each step.
struct StepSchedule {
    const gsn_camera* cameras;  // [view_count]
    const uint8_t* targets;     // view v's target at targets + v * target_stride
    int64_t target_stride;
    const int* views;           // [steps]
    const float* position_lr;   // [steps]
    const float* c1;            // [steps]
    const float* c2;            // [steps]
    const uint32_t* seeds;      // [steps]
    int* cursor;                // next step; advanced by the frame kernel
    int* status;                // sticky GSN_ERR_CAPACITY: schedule, view index or records ran out
    const int* overflow;        // the renderer's record-overflow flag of the previous step
    int steps;
    int view_count;
};
int launch_advance_frame(const StepSchedule& s, StepFrame* frame, cudaStream_t stream);

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
    int* cull_counts;        // [N] optional exact-culling record counts (16 x 16 tiles only), may be null
    int depth_key_shift;     // depth key = float bits >> shift (0: exact order; 8: 24-bit keys, fast forms)
};
// cam_dev (optional): device camera read instead of `cam` (batched form).
// bf16_sh: precision-form parameter layout (10 fp32 rows + 24 rows of bf16 SH pairs).
int launch_project(const float* params, int n, const gsn_camera& cam, const gsn_camera* cam_dev, int sh_degree,
                   bool bf16_sh, const ProjectOutputs& out, cudaStream_t stream);

// Projection with a tile rectangle of tile_w x tile_h pixels (16x16, 16x8 or
// 8x8; the camera's tile counts must match) - the multi-view renderer's sweep.
int launch_project_tiled(const float* params, int n, const gsn_camera& cam, int tile_w, int tile_h, int sh_degree,
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
    uint32_t* digit_total;  // [passes][16 partial copies][256]
    size_t max_blocks;
};
size_t radix_sort_scratch_bytes(int max_count);
RadixSortScratch radix_sort_scratch(void* base, int max_count);
int launch_radix_sort(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt,
                      bool identity_values, int max_count, const int* count_device, int begin_bit,
                      int end_bit, const RadixSortScratch& scratch, bool* result_in_alt,
                      cudaStream_t stream);

// The same sort leaving out every key equal to 0xFFFFFFFF (the culled-Gaussian
// depth key, which sorts last): the first pass drops them and writes the
// number of kept pairs to *kept_device (device int); later passes and the
// sorted output cover only those.
int launch_radix_sort_dropping(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt,
                               bool identity_values, int max_count, const int* count_device, int begin_bit,
                               int end_bit, const RadixSortScratch& scratch, bool* result_in_alt, int* kept_device,
                               cudaStream_t stream);

// Same sort with its scratch in a static device array of the library (no
// allocation); count <= noalloc_sort_max_count(), else GSN_ERR_CAPACITY.
int noalloc_sort_max_count();
int launch_radix_sort_noalloc(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt, int count,
                              int begin_bit, int end_bit, bool* result_in_alt, cudaStream_t stream);

// Exclusive prefix sum of 32-bit integers, in -> out (in-place allowed), n + 1
// outputs with out[n] = total. `gather` (optional) reads in[gather[i]] instead of
// in[i]. Scratch: scan_scratch_bytes(n).
size_t scan_scratch_bytes(int n);
// valid_device (optional): entries from index *valid_device on count as zero.
int launch_exclusive_scan(const int* in, const uint32_t* gather, int* out, int n, void* scratch,
                          cudaStream_t stream, const int* valid_device = nullptr);

// Emit one (tile, gaussian id) record per tile of every visible Gaussian, in
// depth order. record_start[p] is the exclusive scan of tile counts in sorted
// order; records beyond `capacity` are not written and set *overflow.
int launch_emit_records(const uint32_t* sorted_ids, const int* record_start, const int4* rects,
                        int n, int tile_count_x, uint32_t* tile_keys, uint32_t* record_ids,
                        int64_t capacity, int* overflow, cudaStream_t stream);

// Exact tile culling (project.cu): with ProjectOutputs::cull_counts set, the
// projection also counts, per Gaussian, the tiles of its rect whose pixel
// centres the widened alpha >= 1/255 ellipse reaches; launch_emit_records_culled
// emits exactly those records in depth order. Dropped records are ones the blend
// kernels skip at every pixel, so images and gradients are unchanged. A count
// the emitter cannot reproduce sets *overflow to 2 (never expected).
int launch_emit_records_culled(const uint32_t* sorted_ids, const int* record_start, const int4* rects,
                               const float2* means, const float4* conic_opacity, int n, int tile_count_x,
                               uint32_t* tile_keys, uint32_t* record_ids, int64_t capacity, int* overflow,
                               cudaStream_t stream);

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
    // optional: two bit planes of record_words words (plane w at record_warps +
    // w * record_words, cleared by the caller); bit r of plane w is set when a
    // pixel of warp w's strip took record r
    uint32_t* record_warps;
    int64_t record_words;
    bool fast;                     // fast power / exp arithmetic (see raster_common.cuh Power)
    // optional: adds the number of (pixel, record) pairs the blend took (the
    // algorithmic work of the blend and of its backward) to *pair_count; the
    // counting variant of the kernel runs only when it is set
    unsigned long long* pair_count = nullptr;
};
int launch_raster_forward(const RasterForwardArgs& a, cudaStream_t stream);

// ---------------------------------------------------------------- loss
// dL/dimage of 0.8 * L1 + 0.2 * (1 - SSIM) for an fp32 HWC image against a u8
// HWC target. `sums` (optional, 3 doubles, zeroed by the launcher) receives
// sum|I - T|, sum SSIM and sum (I - T)^2 in FP64.
// frame (optional): the target is frame->target instead of `target`.
// fast: products of the moments formed once per input, not once per tap (the
// sums round differently from the reference's kernel; the fast forms only).
int launch_loss_gradient(const float* image, const uint8_t* target, const StepFrame* frame, float* grad, int width,
                         int height, double* sums, cudaStream_t stream, bool fast = false);
// Precision form of the same gradient: the 11x11 window runs as banded-Toeplitz
// GEMMs on the tcgen05 tensor cores with a hi/lo bf16 split and fp32
// accumulation (loss_tc.cu). *status (device) is set to GSN_ERR_TIMEOUT if a
// tensor-core pass never completed.
int launch_loss_gradient_tc(const float* image, const uint8_t* target, const StepFrame* frame, float* grad, int width,
                            int height, double* sums, int* status, cudaStream_t stream);
// FP64 held-out-view metrics (eval.cu): image clamped to [0, 1]; out (device,
// 4 doubles) = PSNR (dB), mean SSIM (11x11 Gaussian window, sigma 1.5, zero
// padding), mean L1, MSE. workspace: eval_metrics_workspace(width, height) bytes.
size_t eval_metrics_workspace(int width, int height);
int launch_eval_metrics(const float* image, const uint8_t* target, int width, int height, double* workspace,
                        double* out, cudaStream_t stream);
// out[0..3] = loss, mean L1, mean SSIM, PSNR (dB) from the sums above.
int launch_finalize_loss(const double* sums, int width, int height, double* out, cudaStream_t stream);

// ---------------------------------------------------------------- backward
struct RasterBackwardArgs {
    const uint32_t* tile_ids;
    const int64_t* tile_offsets;
    const float2* means;
    const float4* conic_opacity;
    const float3* colors;
    const float* image;        // final colours of the forward pass
    const float* image_grad;   // dL/dimage
    const int* contributors;   // per-pixel record bound from the forward pass (optional)
    const uint32_t* record_warps;  // the forward pass's bit planes (optional)
    int64_t record_words;
    bool fast;                 // the forward pass's arithmetic form (must match it)
    gsn_camera cam;
    float* grad_out;           // [N][12] screen-space accumulators, zeroed by the caller
};
int launch_raster_backward(const RasterBackwardArgs& a, cudaStream_t stream);

// ---------------------------------------------------------------- update
struct GaussianUpdateArgs {
    float* params;            // 58 x n SoA, updated in place by Adam
    float* m;                 // Adam first moments (null: no Adam step)
    float* v;                 // Adam second moments
    const float* screen;      // [n][12] from the backward pass
    const int* tile_counts;   // [n] visibility of the frame
    gsn_camera cam;
    int n;
    float lr[6];              // position, log-scale, rotation, opacity, SH DC, SH rest
    float c1, c2;             // Adam bias corrections 1/(1-b1^t), 1/(1-b2^t)
    float* stats;             // optional 2 x n: view-space gradient norm, visible
    float* abs_stats;         // optional 2 x n: norm of the absolute sums, sum|dv|
    float* grad_sums;         // optional density accumulators (all three or none)
    float* abs_sums;
    unsigned int* obs_counts;
    float* grads_out;         // optional 58 x n mapped parameter gradients
    const StepFrame* frame;   // optional: camera, lr[0], c1, c2 and seed come from the device frame
    bool bf16_sh;             // precision-form layout of params, m and v (10 fp32 + 48 bf16 rows)
    uint32_t seed;            // stochastic-rounding seed of the step (precision form)
    bool sparse;              // visibility-masked Adam: Gaussians with tile_counts == 0 keep p, m, v
    // optional with sparse: lazy moment decay. last_step[i] is the step that last
    // updated Gaussian i (0: unknown); a visible Gaussian's moments first decay by
    // b1^k, b2^k for the k steps it skipped, and last_step[i] becomes step
    uint32_t* last_step;
    uint32_t step;
    // optional statistics of the learned density policy (all set or all null),
    // updated for Gaussians visible in the frame: round maximum of the screen
    // radius, round sums of depth and depth^2, and the norms of this step's
    // gradients of mean, log-scale, opacity logit and SH (x, y, z, w)
    const float* radii;       // renderer's 3-sigma pixel radius of the frame
    const float* depths;      // renderer's camera-space depth of the frame
    float* max_radius;
    float* depth_sum;
    float* depth_sq;
    float4* last_grad;
};
int launch_gaussian_update(const GaussianUpdateArgs& a, int sh_degree, cudaStream_t stream);

// Adam history gather after densification: row r of the new moments takes the
// parent's entry, or zero for parent -1 / out of range.
int launch_remap_moments(const int* parents, const float* prev_m, const float* prev_v, float* m, float* v,
                         int prev_count, int count, bool bf16_sh, cudaStream_t stream);

// ---------------------------------------------------------------- spatial order
// Morton keys (30 bits, 10 per axis inside the bounding box of the finite
// means; bounds: 6 ints of device scratch) for a spatial permutation of the
// Gaussians (spatial.cu); the row gather dst[r][i] = src[r][perm[i]] of a
// parameter or moment block in either layout; and parents'[i] = parents[perm[i]]
// (perm[i] itself when parents is null).
int launch_morton_keys(const float* params, int n, int* bounds, uint32_t* keys, cudaStream_t stream);
int launch_gather_gaussians(const float* src, float* dst, const uint32_t* perm, int n, bool bf16_sh,
                            cudaStream_t stream);
int launch_compose_parents(const int* parents, const uint32_t* perm, int n, int* out, cudaStream_t stream);

// ---------------------------------------------------------------- tcgen05
// D (128 x 64 fp32, row-major) = A (128 x 128) * B^T (B: 64 x 128), operands
// fp32 row-major on the device, rounded to bf16 and multiplied on the tensor
// cores; *status is set to GSN_ERR_TIMEOUT if the MMA never completed.
int launch_tc_gemm_selftest(const float* a, const float* b, float* d, int* status, cudaStream_t stream);

}  // namespace gsn
