/*
 * gsn_oracle.h - CPU oracle for the gs-native B200 parity tests.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C, mostly FP64 restatement of the
 * reference's algorithm for the 3DGS training hot path (Naive-q/GS-native:
 * src/core/render/renderer.cu, src/core/solver/solver.cu,
 * src/core/density/density_controller.cu, src/core/knn/knn.cu and the FP64
 * CPU reference test/cpu_reference.h). Only tests/, the smoke check and the
 * benchmark's CPU-baseline leg may call it; the product never links it.
 *
 * Pinning: the oracle is checked against the known-answer values of the
 * reference's own tests (renderer_test.cu, solver_test.cu, density_test.cu,
 * knn_test.cu) by tests/test_oracle_*.py, against FP64 central finite
 * differences of its own forward model, and against the reference's CUDA
 * kernels (compiled unmodified into _ref/libgsref.so) run on the GPU by the
 * -m gpu tests on identical inputs.
 */
#ifndef GSN_ORACLE_H
#define GSN_ORACLE_H

#include <stdint.h>

#include "../include/gsn_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Projected Gaussian (renderer.cu:108-221; cpu_reference.h:45-85), FP64. */
typedef struct orc_proj {
    int visible;
    int rect[4];        /* tile rect [x0, y0, x1, y1) */
    double depth;       /* camera z */
    double u, v;        /* pixel centre */
    double cov[3];      /* 2D covariance a, b, c incl. the 0.3 low-pass */
    double conic[3];    /* inverse of cov */
    double opacity;
    double radius;
    double rgb[3];      /* colour after the lower clamp */
    double rgb_raw[3];  /* SH value + 0.5 before the clamp */
} orc_proj;

/* Per-row learning rates of the Adam step (solver.cu:666-681). */
typedef struct orc_lr {
    double position, scale, rotation, opacity, sh_dc, sh_rest;
} orc_lr;

/* Projection of n Gaussians from the 58 x n SoA block. */
void orc_project(const float* params, int n, const gsn_camera* cam, int sh_degree, orc_proj* out);

/* Integer tile-record ordering of the reference (renderer.cu:223-271, 541-563):
 * keys (tile << 32 | depth bits) written in id order, stably sorted, then
 * per-tile offsets. Inputs are per Gaussian: depth float bits, rect int4 and
 * tile count (0 = culled). out_ids must hold sum(counts) entries, out_offsets
 * tile_count + 1. Returns the record count. */
int64_t orc_sort_records(const uint32_t* depth_bits, const int* rects, const int* counts, int n,
                         int tile_count_x, int tile_count_y, int32_t* out_ids, int64_t* out_offsets);

/* Depth-ordered per-tile lists from FP64 projections: tile t holds the visible
 * Gaussians whose rect covers it, ordered by (depth, id) (cpu_reference.h:36-41).
 * Allocates *offsets (tiles + 1) and *ids; free with orc_free. */
void orc_tile_lists(const orc_proj* p, int n, const gsn_camera* cam, int64_t** offsets, int32_t** ids);
void orc_free(void* ptr);

/* FP64 alpha blending over the tile lists (renderer.cu:273-338 with the
 * thresholds of cpu_reference.h:86-108). image: HWC double. Optional outputs:
 * final transmittance per pixel, contributors (records consumed before the last
 * contribution). Tiles [tile_begin, tile_end) only (all when tile_end <= 0). */
void orc_render(const orc_proj* p, const gsn_camera* cam, const int64_t* offsets, const int32_t* ids,
                const double* background, double* image, double* final_t, int* contributors, int tile_begin,
                int tile_end);

/* Loss 0.8 * L1 + 0.2 * (1 - SSIM), 11x11 Gaussian window sigma 1.5, zero padding
 * (cpu_reference.h:120-152). target: u8 HWC. Rows [row_begin, row_end) only
 * contribute to the sums when row_end > 0 (normalised by the full image). */
double orc_loss(const double* image, const uint8_t* target, int width, int height);

/* Held-out-view metrics: image clamped to [0, 1]; out = PSNR (dB), mean SSIM
 * (11x11, sigma 1.5, zero padding), mean L1, MSE. FP64. */
void orc_eval_metrics(const double* image, const uint8_t* target, int width, int height, double* out);

/* Analytic dLoss/dimage of orc_loss (the quantity of solver.cu:26-168), FP64. */
void orc_loss_gradient(const double* image, const uint8_t* target, int width, int height, double* gradient,
                       int row_begin, int row_end);

/* Screen-space backward (solver.cu:325-466): per Gaussian 9 rows
 * [du, dv, dcov_a, dcov_b, dcov_c, dlogit, dr, dg, db] and 2 absolute rows
 * [|du|, |dv|] summed over pixels; arrays are zeroed by the caller
 * (grad9: 9 x n, abs2: 2 x n, row-major by field). */
void orc_backward(const orc_proj* p, int n, const gsn_camera* cam, const int64_t* offsets, const int32_t* ids,
                  const double* image, const double* image_gradient, double* grad9, double* abs2,
                  int tile_begin, int tile_end);

/* View-space statistics (solver.cu:468-490): stats 2 x n (norm, visible),
 * abs_stats n (norm of the absolute sums). */
void orc_projection_statistics(const orc_proj* p, int n, const gsn_camera* cam, const double* grad9,
                               const double* abs2, double* stats, double* abs_stats);

/* Chain rule to the 58 parameters (solver.cu:185-323, 492-623), FP64.
 * grad58: 58 x n, fully written. */
void orc_map_gradients(const float* params, int n, const gsn_camera* cam, int sh_degree, const double* grad9,
                       double* grad58);

/* Adam step (solver.cu:651-689, bias corrections 912-914) on FP64 state;
 * params is updated in double and m, v are 58 x n. `step` is 1-based. */
void orc_adam(double* params, double* m, double* v, const double* grad58, int n, const orc_lr* lr,
              uint64_t step);

/* Densification decision of density_controller.cu:60-116 for every Gaussian:
 * out4 = (keep, clone, split_sampled, split_keep) as ints (4 x n, interleaved). */
void orc_density_counts(const float* params, int n, const float* gradient_sums, const float* absolute_sums,
                        const uint32_t* observation_counts, float gradient_threshold, float split_threshold,
                        float min_opacity, float max_world_size, int prune_large,
                        float absolute_gradient_threshold, int* out4);

/* Compaction of density_controller.cu:118-278 given the decisions and the normal
 * samples (6 per split-sampled Gaussian, laid out as the reference's samples
 * buffer). Writes the new 58 x new_count block, parent ids (source Gaussian of
 * every output) and history parent ids (-1 for new Gaussians). Returns
 * new_count. */
int orc_density_apply(const float* params, int n, const int* counts4, const float* samples, float* out_params,
                      int* parent_ids, int* history_parent_ids);

/* Exhaustive 3-NN: mean of the up to 3 smallest squared distances (FP64; 0 when
 * n < 2) and the neighbour indices (-1 when missing), knn_test.cu:23-32. */
void orc_knn3(const float* points, int n, double* mean_dist2, int* neighbors);

/* Threads used by the OpenMP loops of the oracle. */
int orc_set_threads(int threads);

#ifdef __cplusplus
}
#endif

#endif /* GSN_ORACLE_H */
