/*
 * gsn.h - C ABI of the gs-native B200 3D Gaussian Splatting training hot path.
 *
 * Plain C: pointers, sizes and opaque handles only. Every entry point returns a
 * gsn status (0 = GSN_OK, negative = error, see gsn_types.h) and never throws.
 * Device pointers are CUDA device addresses; `stream` is a cudaStream_t passed as
 * void* (NULL = legacy default stream). Invalid arguments return
 * GSN_ERR_INVALID_ARGUMENT without side effects, like the reference's `false`
 * returns (e.g. renderer.cu:379-381, 451-454; density_controller.cu:473-481).
 *
 * The handle-based objects wrap the C++ drop-in classes of the gs_native
 * namespace (same semantics as the reference classes they replace); the
 * stateless stage functions expose single kernels for FFI callers and for the
 * parity tests.
 */
#ifndef GSN_H
#define GSN_H

#include <stddef.h>
#include <stdint.h>

#include "gsn_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ library */

/* Library version string. */
const char* gsn_version(void);

/* Synchronous byte copy between host/device memory (cudaMemcpyDefault). For FFI
 * callers without their own CUDA bindings. */
int gsn_memcpy(void* dst, const void* src, size_t bytes);

/* Asynchronous byte copy on `stream` (cudaMemcpyDefault); host memory should
 * be pinned for the copy to overlap. */
int gsn_memcpy_async(void* dst, const void* src, size_t bytes, void* stream);

/* Raw device allocation (cudaMalloc / cudaFree). Parameter blocks handed to
 * gsn_density_control change owner (the controller keeps the caller's old block
 * and frees it itself), so they must come from this allocator or cudaMalloc. */
int gsn_device_alloc(size_t bytes, void** out);
int gsn_device_free(void* ptr);

/* Blocks until all work on `stream` is done. */
int gsn_stream_synchronize(void* stream);

/* Number of this library's kernel launches since load (process-wide). */
uint64_t gsn_kernel_launch_count(void);

/* Programmatic dependent launch of the training step's kernels (gs-native
 * extension, process-wide, on by default): on an eager stream each step kernel
 * is launched with programmatic stream serialization and waits for its
 * predecessor on the device, so a grid's CTAs are scheduled while the one
 * before it drains. Launches captured into a CUDA graph never use it. Results
 * are the same either way. */
int gsn_set_programmatic_launch(int enabled);

/* Stage profiler: when enabled, stage boundaries record CUDA events on the
 * stream of the stage; gsn_profile_collect synchronises and writes the device
 * milliseconds per stage since the last collect into ms[0..count) (stage
 * names via gsn_stage_name). */
int gsn_profile_enable(int enabled);
int gsn_profile_collect(double* ms, int count);
const char* gsn_stage_name(int stage);
int gsn_stage_count(void);

/* ------------------------------------------------------------------ ordering
 * Stable LSD radix sort of (uint32 key, uint32 value) pairs: the ordering
 * primitive of the tile records, used where the reference calls
 * cub::DeviceRadixSort::SortPairs (renderer.cu:541-563). Keys are sorted on bits
 * [begin_bit, end_bit) (end_bit - begin_bit <= 32), ties keep their input order.
 * The data ping-pongs between (keys, values) and (keys_alt, values_alt); on
 * return *result_in_alt (host int) tells which pair holds the sorted output.
 * All arrays are device memory of `count` elements.
 */

/* Device workspace bytes gsn_sort_pairs needs for up to max_count pairs. */
int gsn_sort_pairs_workspace(int max_count, size_t* bytes);

/* Sorts with a caller-provided device workspace of gsn_sort_pairs_workspace bytes. */
int gsn_sort_pairs(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt, int count,
                   int begin_bit, int end_bit, void* workspace, size_t workspace_bytes, int* result_in_alt,
                   void* stream);

/* Allocation-free variant of gsn_sort_pairs (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory themselves or let a library do
 * it: code running under an allocator that owns the whole device budget (a
 * framework's caching allocator or a fixed arena, where a stray cudaMalloc would
 * exceed the budget or fragment the pool), and latency-critical loops that cannot
 * take the device-wide synchronisation that cudaMalloc/cudaFree imply. The caller
 * still passes all four key/value arrays; the sort's histogram scratch lives in a
 * static device array inside the library, sized for at most
 * GSN_SORT_NOALLOC_MAX_COUNT pairs (5.7 MB, reserved on every GPU that loads the
 * library until the process exits). Larger counts return GSN_ERR_CAPACITY and
 * launch nothing. The function calls no cudaMalloc/cudaFree.
 *
 * The first call on a device looks up the scratch array's device address
 * (cudaGetSymbolAddress, with that device current); make that first call before
 * any stream capture. All calls share the one array and it keeps the previous
 * call's contents (the sort clears what it needs): calls that overlap on the GPU,
 * on different streams of the same device, race on it and must be serialised by
 * the caller. Results are identical to gsn_sort_pairs. */
#define GSN_SORT_NOALLOC_MAX_COUNT 16777216
int gsn_sort_pairs_noalloc(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt, int count,
                           int begin_bit, int end_bit, int* result_in_alt, void* stream);

/* Exclusive prefix sum of `count` device ints, the record scan of the ordering
 * (gs-native extension; the reference's Render runs cub::DeviceScan::
 * ExclusiveSum in place over its tile counts, renderer.cu:465-483): out[i] = the sum of
 * the entries before i, out[count] = the total, where entry j is
 * in[gather ? gather[j] : j] for j < *valid (device int; all `count` when
 * valid is null) and zero from there on. `out` holds count + 1 ints; in == out
 * is allowed without `gather`. One pass with decoupled look-back. Device
 * workspace: gsn_exclusive_scan_workspace bytes. */
int gsn_exclusive_scan_workspace(int max_count, size_t* bytes);
int gsn_exclusive_scan(const int* in, const uint32_t* gather, int* out, int count, const int* valid,
                       void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------ 3-NN
 * LBVH 3-nearest-neighbour search (replaces ComputeMeanDist2Cuda, reference
 * src/core/knn/knn.h:9 and knn.cu:180-255). points: device float[3 * count]
 * (xyz); mean_dist2: device float[count], the mean of the up to three smallest
 * squared distances (0 when count < 2); neighbors: optional device
 * int[3 * count] with the neighbour indices (ties to the smaller index, -1 when
 * missing); workspace: device memory of gsn_knn3_workspace bytes. */
int gsn_knn3_workspace(int count, size_t* bytes);
int gsn_knn3(const float* points, int count, float* mean_dist2, int* neighbors, void* workspace, void* stream);

/* Host-to-host convenience form of the same search (allocates internally). */
int gsn_knn3_host(const float* points, int count, float* mean_dist2, int* neighbors);

/* ------------------------------------------------------------------ renderer
 * Replaces gs_native::Renderer (reference src/core/render/renderer.h:10-89).
 */
typedef struct gsn_renderer gsn_renderer;

int gsn_renderer_create(gsn_renderer** out);
int gsn_renderer_destroy(gsn_renderer* r);
int gsn_renderer_set_stream(gsn_renderer* r, void* stream);

/* Renderer::Render (renderer.h:21-26; renderer.cu:359-372): project the 58 x count
 * SoA `params` (device), build the depth-ordered per-tile lists and blend into
 * `image` (device, fp32 HWC RGB, width*height*3). `background` is a host float[3].
 * sh_degree is clamped to [0, 3]. */
int gsn_renderer_render(gsn_renderer* r, const float* params, int count, const gsn_camera* camera,
                        const float* background, float* image, int sh_degree);

/* Device pointers owned by the renderer, valid until the next render call.
 * Getters of renderer.h:28-54 plus the extensions documented in renderer.h. */
typedef struct gsn_renderer_buffers {
    const float* means;            /* float2[count]: (u, v) */
    const float* conic_opacity;    /* float4[count]: (a, b, c, opacity) */
    const float* colors;           /* float3[count] */
    const float* depths;           /* float[count], valid where tile_counts > 0 */
    const int* rects;              /* int4[count]: tile rect [x0, y0, x1, y1), valid where tile_counts > 0 */
    const int* tile_counts;        /* int[count] */
    const float* radii;            /* float[count], 0 when culled */
    const int* tile_gaussian_ids;  /* int[record_count] sorted by (tile, depth, id) */
    const int64_t* tile_offsets;   /* int64[tiles + 1] */
    const int* contributors;       /* int[width * height]: records consumed per pixel */
    const int* record_count;       /* device int */
    const int* overflow;           /* device int, nonzero when a fixed capacity overflowed */
    int64_t record_count_host;     /* host copy (grow mode) */
    int gaussian_capacity;
    int tile_capacity;
} gsn_renderer_buffers;
int gsn_renderer_get_buffers(gsn_renderer* r, gsn_renderer_buffers* out);

/* Renderer::GetRecordOffsets (renderer.h:44-46): exclusive scan of tile counts in
 * id order, count + 1 entries. */
int gsn_renderer_record_offsets(gsn_renderer* r, const int** out);

/* Fixed record capacity (0 = grow on demand, the reference behaviour). */
int gsn_renderer_set_record_capacity(gsn_renderer* r, int64_t records);
/* Precision form (gs-native extension): `enabled` selects the parameter layout
 * of 10 fp32 geometry rows followed by the 48 SH coefficients in bf16 as 24
 * rows of pairs (34 rows of 32-bit words of stride count; SH coefficient 2r of
 * Gaussian i in the low 16 bits of word r * count + i of the SH rows, 2r + 1 in
 * the high 16 bits). The same switch exists on the solver (parameters and Adam
 * moments; SH updates use stochastic rounding; switching drops the history)
 * and on the density controller. */
int gsn_renderer_set_bf16_sh(gsn_renderer* r, int enabled);
/* Exact tile culling (gs-native extension): emit only the records whose tile
 * the (widened) alpha >= 1/255 ellipse of the Gaussian reaches, instead of
 * every tile of its 3-sigma rectangle (renderer.cu:223-245). Images and
 * gradients are unchanged; per-tile lists are the reference's minus records
 * that never contribute. Tile counts / record offsets keep the rectangle
 * counts (the solver's visibility statistic, solver.cu:484). */
int gsn_renderer_set_exact_culling(gsn_renderer* r, int enabled);
/* Fast blend arithmetic (gs-native extension): the per-pixel Gaussian power in
 * Horner form with per-record terms hoisted and the hardware exp2
 * approximation, instead of the expression and expf of renderer.cu:300-305.
 * Images move by a few ulps; the solver's backward pass follows the setting. */
int gsn_renderer_set_fast_blend(gsn_renderer* r, int enabled);
/* Measurement hook (gs-native extension, no reference counterpart): while
 * device_counter (device unsigned long long) is set, each render adds the
 * number of (pixel, record) pairs its blend took to it; NULL turns it off. */
int gsn_renderer_set_pair_counter(gsn_renderer* r, unsigned long long* device_counter);


/* ------------------------------------------------------------------ solver
 * Replaces gs_native::Solver (reference src/core/solver/solver.h:11-68).
 * A solver is paired with the renderer whose last frame it differentiates.
 */
typedef struct gsn_solver gsn_solver;

int gsn_solver_create(gsn_solver** out);
int gsn_solver_destroy(gsn_solver* s);
int gsn_solver_set_stream(gsn_solver* s, void* stream);

/* Solver::Iterate (solver.h:19-26; solver.cu:702-720): loss gradient of `image`
 * (device fp32 HWC, the renderer's output) against `target` (device u8 HWC),
 * backward through the renderer's frame, chain rule and one Adam step on the
 * 58 x count device block `params`. */
int gsn_solver_iterate(gsn_solver* s, const gsn_camera* camera, gsn_renderer* renderer, const float* image,
                       const uint8_t* target, float* params, int count, float position_lr, int sh_degree);

/* Solver::ResetOpacityHistory (solver.cu:722-733). */
int gsn_solver_reset_opacity_history(gsn_solver* s);

/* Solver::RemapGaussians (solver.cu:761-835): parent_ids (device, may be NULL)
 * maps every new Gaussian to the old index whose Adam history it inherits
 * (-1 = fresh history). */
int gsn_solver_remap(gsn_solver* s, const int* parent_ids, int count);

/* GetProjectionStatistics / GetAbsoluteProjectionStatistics (solver.h:35-41):
 * device float[2 * count] each. */
int gsn_solver_statistics(gsn_solver* s, const float** stats, const float** absolute_stats);

/* Learning rates of the non-position groups (reference defaults: scale 0.005,
 * rotation 0.001, opacity 0.025, SH DC 0.0025, SH rest 0.0025 / 20). */
int gsn_solver_set_learning_rates(gsn_solver* s, float scale, float rotation, float opacity, float sh_dc,
                                  float sh_rest);

/* Enables the FP64 loss reduction; gsn_solver_loss then copies
 * [loss, mean L1, mean SSIM, PSNR dB] of the last iterate to `out` (host). */
int gsn_solver_set_compute_loss(gsn_solver* s, int enabled);
int gsn_solver_set_bf16_sh(gsn_solver* s, int enabled);
/* The L1+SSIM gradient on the tcgen05 tensor cores (banded-Toeplitz GEMMs,
 * hi/lo bf16 split, fp32 accumulation): on with the precision form, switchable
 * on its own. gsn_solver_status synchronises and returns GSN_OK or
 * GSN_ERR_TIMEOUT (a tensor-core pass did not complete). */
int gsn_solver_set_tensor_core_loss(gsn_solver* s, int enabled);
int gsn_solver_status(gsn_solver* s, int* status);
int gsn_solver_loss(gsn_solver* s, double* out);
int gsn_solver_loss_device(gsn_solver* s, const double** out);

/* Visibility-masked (sparse) Adam (gs-native extension): Gaussians with no tile
 * in the frame keep parameters and moments; the reference updates all
 * 58 x N every iteration (solver.cu:912-915). */
int gsn_solver_set_sparse_adam(gsn_solver* s, int enabled);
/* Lazy moment decay for the sparse update (gs-native extension, off by default):
 * a Gaussian that skipped k steps has its moments scaled by 0.9^k and 0.999^k
 * before its next update, the decay k dense zero-gradient steps would apply.
 * Needs sparse Adam; eager steps only (a step through a CUDA graph fails). */
int gsn_solver_set_lazy_moment_decay(gsn_solver* s, int enabled);
/* Stage entry points of Iterate for parity tests and partial pipelines:
 * dL/dimage into the solver's buffer (device float[pixels * 3] via *out);
 * screen-space gradients ([count][12] floats via *out); mapped parameter
 * gradients (58 x count) into `grads_out` without an Adam step. */
int gsn_solver_image_gradients(gsn_solver* s, const gsn_camera* camera, const float* image, const uint8_t* target,
                               const float** out);
int gsn_solver_screen_gradients(gsn_solver* s, const gsn_camera* camera, gsn_renderer* renderer,
                                const float* image, const float* params, int count, const float** out);
int gsn_solver_map_gradients(gsn_solver* s, const gsn_camera* camera, gsn_renderer* renderer, float* params,
                             int count, int sh_degree, float* grads_out);

/* Adam state (device, 58 x count each) and the step counter. */
int gsn_solver_moments(gsn_solver* s, float** first, float** second, uint64_t* iteration);


/* ------------------------------------------------------------------ density
 * Replaces gs_native::DensityController (reference
 * src/core/density/density_controller.h:9-83).
 */
typedef struct gsn_density gsn_density;

int gsn_density_create(gsn_density** out);
int gsn_density_destroy(gsn_density* d);
int gsn_density_set_stream(gsn_density* d, void* stream);

/* Initialize (density_controller.cu:410-438). */
int gsn_density_initialize(gsn_density* d, int count, int capacity);

/* AccumulateStatistics(statistics, absolute_statistics, count)
 * (density_controller.cu:613-631): device float[2 * count] + float[count]. */
int gsn_density_accumulate(gsn_density* d, const float* statistics, const float* absolute_statistics, int count);

/* AccumulateStatistics(gradients, radii, ids, observations)
 * (density_controller.cu:440-459): per-observation 2D gradients. */
int gsn_density_accumulate_observations(gsn_density* d, const float* gradients, const float* radii, const int* ids,
                                        int observations);

/* ResetOpacity (density_controller.cu:633-647). */
int gsn_density_reset_opacity(gsn_density* d, float* params, int stride, float max_opacity);

/* ControlDensity (density_controller.cu:461-611). On success *params / *count
 * receive the new parameter block (owned by the caller from now on) and the
 * caller's previous block becomes the controller's spare (ownership ping-pong);
 * all pruned: *params = NULL, *count = 0. changes (optional host int[2]) =
 * {added, removed}. */
int gsn_density_control(gsn_density* d, float** params, int* count, float scene_extent, float gradient_threshold,
                        float percent_dense, float min_opacity, float max_screen_size, unsigned long long seed,
                        int* changes, float absolute_gradient_threshold);

/* GetHistoryParentIds / GetGaussianCount (control block) / GetParentIds (device). */
int gsn_density_buffers(gsn_density* d, const int** history_parent_ids, const int** control, const int** parent_ids);

/* Cap on the Gaussian count (0 = unlimited, the reference behaviour): additions
 * beyond the cap are dropped in id order. */
int gsn_density_set_max_gaussians(gsn_density* d, int max_gaussians);
int gsn_density_set_bf16_sh(gsn_density* d, int enabled);

/* The normal samples of the last ControlDensity (device float[6 * sampled]) and
 * the accumulated statistics (device float[capacity] x2, uint[capacity]). */
int gsn_density_internals(gsn_density* d, const float** samples, float** gradient_sums, float** absolute_sums,
                          unsigned int** observation_counts);


/* ------------------------------------------------------------------ trainer
 * Replaces gs_native::GaussianSplatting (reference
 * src/core/gaussian_splatting.h:14-53), without OpenCV: the scene is camera
 * parameters, host u8 HWC images and a host point cloud. Defaults of
 * gsn_training_options_default equal the reference's hard-coded schedule
 * (gaussian_splatting.cpp:130-198, 262-287; solver.cu:666-681).
 */
typedef struct gsn_training_options {
    int sh_degree_interval;          /* 1000 */
    int max_sh_degree;               /* 3 */
    float position_lr_init;          /* 1.6e-4 (times the scene extent) */
    float position_lr_final;         /* 1.6e-6 */
    int position_lr_steps;           /* 30000 */
    float lr_scale, lr_rotation, lr_opacity, lr_sh_dc, lr_sh_rest; /* 0.005 0.001 0.025 0.0025 0.0025/20 */
    int densify_from;                /* 500 */
    int densify_until;               /* 15000 */
    int densify_interval;            /* 100 */
    float gradient_threshold;        /* 2e-4 */
    float absolute_gradient_threshold; /* 8e-4 */
    float percent_dense;             /* 0.01 */
    float min_opacity;               /* 0.005 */
    int prune_large_after;           /* 3000 */
    int opacity_cap_interval;        /* 500 */
    float opacity_cap;               /* 0.8 */
    int opacity_reset_interval;      /* 3000 */
    float opacity_reset;             /* 0.01 */
    float background[3];             /* 0 0 0 */
    int max_gaussians;               /* 0 = unlimited */
    unsigned long long density_seed; /* 0 */
    float initial_opacity;           /* 0.1 */
    /* gs-native extensions (0 = reference behaviour) */
    int precision;                   /* 1: precision form - SH and its Adam moments stored in bf16 */
    int graph;                       /* 1: iterations after densify_until run as CUDA-graph replays */
    int learned_density;             /* 1: the learned policy (gsn_trainer_set_density_mlp) proposes actions */
    float learned_confidence;        /* 0.9: softmax probability needed to override the threshold rule */
    int log_density;                 /* 1: keep the last control step's statistics (gsn_trainer_density_log) */
    int exact_culling;               /* 1: exact tile culling in the training renderer (gsn_renderer_set_exact_culling) */
    int sparse_adam;                 /* 1: visibility-masked Adam (gsn_solver_set_sparse_adam) */
    int spatial_order;               /* 1: Morton order of the Gaussians after init and every density step */
    int fast_blend;                  /* 1: fast blend arithmetic in the training renderer (gsn_renderer_set_fast_blend) */
    int fp32_ssim;                   /* 1: the precision form keeps the fp32 SSIM gradient kernel */
} gsn_training_options;

int gsn_training_options_default(gsn_training_options* out);

typedef struct gsn_trainer gsn_trainer;
int gsn_trainer_create(gsn_trainer** out);
int gsn_trainer_destroy(gsn_trainer* t);
int gsn_trainer_set_stream(gsn_trainer* t, void* stream);
/* Initialize (gaussian_splatting.cpp:23-128): images[k] is a host u8 HWC image
 * of cameras[k]; points / colors are host float[3 * point_count]. */
int gsn_trainer_initialize(gsn_trainer* t, const gsn_camera* cameras, const uint8_t* const* images,
                           int camera_count, const float* points, const float* colors, int point_count,
                           const gsn_training_options* options);
/* Train (gaussian_splatting.cpp:130-198). */
int gsn_trainer_train(gsn_trainer* t, int iterations);
/* The trainer's solver: gsn_solver_set_lazy_moment_decay (needs the sparse_adam
 * option and graph = 0). */
int gsn_trainer_set_lazy_moment_decay(gsn_trainer* t, int enabled);
/* Render into a device fp32 HWC image (gaussian_splatting.cpp:200-232). */
int gsn_trainer_render(gsn_trainer* t, const gsn_camera* camera, float* image);
/* Mean PSNR / loss over views with host u8 HWC images (FP64 reductions). */
int gsn_trainer_evaluate(gsn_trainer* t, const gsn_camera* cameras, const uint8_t* const* images, int count,
                         double* psnr, double* loss);
/* Mean FP64 PSNR (dB), SSIM (11x11 window), L1 and loss over held-out views
 * (host u8 HWC images); outputs may be null. gs-native extension. */
int gsn_trainer_evaluate_metrics(gsn_trainer* t, const gsn_camera* cameras, const uint8_t* const* images, int count,
                                 double* psnr, double* ssim, double* l1, double* loss);
/* FP64 held-out-view metrics of one rendered view on the GPU (gs-native
 * extension): image (device fp32 HWC) clamped to [0, 1] against the device u8
 * HWC target; out (host, 4 doubles) = PSNR (dB), mean SSIM (11x11 Gaussian
 * window, sigma 1.5, zero padding), mean L1, MSE. Synchronises the stream. */
int gsn_eval_metrics(const float* image, const uint8_t* target, int width, int height, double* out, void* stream);
/* Save to / load from a Gaussian PLY (gaussian_splatting.cpp:234-260). */
int gsn_trainer_save(gsn_trainer* t, const char* path);
int gsn_trainer_load(gsn_trainer* t, const char* path);
/* Current device parameter block and schedule state. */
int gsn_trainer_state(gsn_trainer* t, float** params, int* count, int* completed, int* sh_degree,
                      float* scene_extent);

/* ------------------------------------------------------------------ batched form
 * gs-native extension (the reference runs every stage from the host and reads
 * the record count back each frame, renderer.cu:480-500): one CUDA graph holds
 * a whole training iteration (projection, sorts, forward, loss, backward,
 * Adam) over a fixed record capacity with device-side counts, and a device
 * schedule supplies each replay's view, position learning rate and Adam step.
 *
 * gsn_graph_capture: the renderer and solver are bound to the graph (and their
 * stream set to `stream`) until gsn_graph_destroy; `params` / `count` must stay
 * the same block. cameras[0..camera_count) share one resolution; view v's u8
 * HWC target is resident at device_targets + v * target_stride.
 * gsn_graph_run: `steps` replays, view views[k] with position lr
 * position_lrs[k] (host arrays); asynchronous on the capture stream.
 * gsn_graph_check: synchronises; GSN_ERR_CAPACITY if any step since the last
 * check exceeded record_capacity tile records. */
typedef struct gsn_graph gsn_graph;
int gsn_graph_create(gsn_graph** out);
int gsn_graph_destroy(gsn_graph* g);
int gsn_graph_capture(gsn_graph* g, gsn_renderer* renderer, gsn_solver* solver, float* params, int count,
                      const gsn_camera* cameras, int camera_count, const uint8_t* device_targets,
                      size_t target_stride, const float* background, float* device_image, int sh_degree,
                      int64_t record_capacity, void* stream);
int gsn_graph_run(gsn_graph* g, const int* views, const float* position_lrs, int steps);
int gsn_graph_check(gsn_graph* g);
int gsn_graph_launches_per_step(gsn_graph* g, int* out);

/* ------------------------------------------------------------------ multi-view renderer
 * gs-native extension: `count` cameras of any resolutions rendered into device
 * fp32 HWC images (images[v] points at width * height * 3 floats) with one
 * persistent blend launch over all (view, tile) work items. Configuration:
 * tile 16x16, 16x8 or 8x8; 64, 128 or 256 threads per tile (at least one
 * pixel row per thread); sort key width 32 (depth pre-sort + tile bits), 48
 * (tile|depth over 32 + log2 T bits) or 64. gsn_multiview_autotune times every
 * valid configuration on the given views, keeps the fastest and writes up to
 * max_results rows of {tile_w, tile_h, threads, key_bits, ms} to results. */
typedef struct gsn_multiview gsn_multiview;
int gsn_multiview_create(gsn_multiview** out);
int gsn_multiview_destroy(gsn_multiview* m);
int gsn_multiview_set_stream(gsn_multiview* m, void* stream);
int gsn_multiview_set_config(gsn_multiview* m, int tile_w, int tile_h, int threads, int key_bits);
int gsn_multiview_get_config(gsn_multiview* m, int* tile_w, int* tile_h, int* threads, int* key_bits);
int gsn_multiview_render(gsn_multiview* m, const float* params, int count, const gsn_camera* cameras, int views,
                         float* const* images, const float* background, int sh_degree);
int gsn_multiview_autotune(gsn_multiview* m, const float* params, int count, const gsn_camera* cameras, int views,
                           float* const* images, const float* background, int sh_degree, int repeats,
                           float* results, int max_results, int* result_count);

/* ------------------------------------------------------------------ tensor cores
 * Self-test of the tcgen05 path used by the precision form's SSIM filter
 * (gs-native extension): d (128 x 64 fp32, row-major) = a (128 x 128) * b^T
 * (b: 64 x 128), all device pointers, operands rounded to bf16, accumulated in
 * fp32 tensor memory. Synchronises; GSN_ERR_TIMEOUT if the MMA did not finish. */
int gsn_tc_gemm_selftest(const float* a, const float* b, float* d, void* stream);

/* Resumable checkpoint (gs-native extension): parameters in their stored
 * layout, Adam moments and step, density statistics, iteration, camera order
 * and cursor. Load after gsn_trainer_initialize with the same scene/options. */
int gsn_trainer_save_checkpoint(gsn_trainer* t, const char* path);
int gsn_trainer_load_checkpoint(gsn_trainer* t, const char* path);

/* Learned density policy of the trainer: MLP weights (host, GSN_MLP_PARAMS
 * floats; used when options.learned_density is set) and the log of the last
 * density-control step (device pointers valid until the next step):
 * features [before][16], decisions [before] (0 keep, 1 clone, 2 split,
 * 3 prune), parents [after] (source index of each output Gaussian). */
int gsn_trainer_set_density_mlp(gsn_trainer* t, const float* weights);
int gsn_trainer_density_log(gsn_trainer* t, const float** features, const int8_t** decisions, const int** parents,
                            int* before, int* after, int* steps, int* iteration);

/* ------------------------------------------------------------------ learned density MLP
 * gs-native extension: 16 statistics -> 64 -> 64 -> {keep, clone, split,
 * prune}, ReLU, fp16 working weights, fp32 arithmetic; trained on the GPU by
 * the library's own fused forward/backward kernels (full-batch Adam on the
 * weighted mean cross-entropy). Device arrays: features [n][16] float, labels
 * [n] int (0..3), sample weights [n] float, actions [n] int8, probs [n][4]. */
#define GSN_MLP_PARAMS 5508
typedef struct gsn_mlp gsn_mlp;
int gsn_mlp_create(gsn_mlp** out);
int gsn_mlp_destroy(gsn_mlp* m);
int gsn_mlp_initialize(gsn_mlp* m, unsigned long long seed);
int gsn_mlp_set_weights(gsn_mlp* m, const float* host_weights);
int gsn_mlp_get_weights(gsn_mlp* m, float* host_weights);
int gsn_mlp_gradients(gsn_mlp* m, const float* features, const int* labels, const float* weights, int n,
                      float* host_grad, double* loss);
int gsn_mlp_train(gsn_mlp* m, const float* features, const int* labels, const float* weights, int n, int steps,
                  float lr, double* loss);
int gsn_mlp_infer(gsn_mlp* m, const float* features, int n, float confidence, int8_t* actions, float* probs);

/* ------------------------------------------------------------------ PLY
 * WriteGaussiansPly / ReadGaussiansPly (reference src/io/data_io.cpp:420-590)
 * on a host 58 x count SoA block. */
int gsn_ply_write(const char* path, const float* params, int count);
int gsn_ply_read_count(const char* path, int* count);
int gsn_ply_read(const char* path, float* params, int count);

/* ------------------------------------------------------------------ spatial order
 * gs-native extension: a Morton-order permutation of the Gaussians (30-bit keys
 * of the means inside their bounding box; ties keep id order) and the row
 * gather that applies it to a parameter or Adam-moment block (dst[r][i] =
 * src[r][perm[i]], 58 fp32 rows, or the precision layout when bf16_sh). No
 * rendered or trained value depends on the order; locality does. Device
 * pointers; perm holds count uint32. */
int gsn_spatial_permutation(const float* params, int count, uint32_t* perm, void* stream);
int gsn_gather_gaussians(const float* src, float* dst, const uint32_t* perm, int count, int bf16_sh, void* stream);

/* ------------------------------------------------------------------ COLMAP scene
 * ReadColmapScene (reference src/io/data_io.cpp:328-418) without OpenCV:
 * sparse/0/{cameras,images,points3D}.bin (one PINHOLE camera), images
 * pre-decoded to binary PPM (P6) under images/ (images/<name> when it is a PPM,
 * else images/<name without extension>.ppm), integer downscale by block
 * averaging. Images sorted by name; every 8th is a test view. Cameras carry
 * near 0.2, far FLT_MAX and 16x16 tiles. split: 0 train, 1 test. Image
 * pointers are host u8 HWC and live as long as the scene. */
typedef struct gsn_scene gsn_scene;
int gsn_scene_read_colmap(const char* scene_dir, int downscale, gsn_scene** out);
int gsn_scene_destroy(gsn_scene* s);
int gsn_scene_counts(const gsn_scene* s, int* train, int* test, int* points);
int gsn_scene_view(const gsn_scene* s, int split, int index, gsn_camera* camera, const uint8_t** image,
                   const char** name);
int gsn_scene_points(const gsn_scene* s, const float** positions, const float** colors);
/* Binary PPM (P6, maxval 255) and PNG (8-bit RGB, uncompressed deflate) writers. */
int gsn_image_write_ppm(const char* path, const uint8_t* rgb, int width, int height);
int gsn_image_write_png(const char* path, const uint8_t* rgb, int width, int height);

#ifdef __cplusplus
}
#endif

#endif /* GSN_H */
