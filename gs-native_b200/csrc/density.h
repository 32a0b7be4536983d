// Launchers of the density-control kernels (density.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "kernels.h"

namespace gsn {

struct DensityThresholds {
    float gradient_threshold;           // mean view-space gradient for densification
    float split_threshold;              // percent_dense * scene extent
    float min_opacity;
    float max_world_size;               // 0.1 * scene extent
    float absolute_gradient_threshold;  // > 0: splits use the absolute statistic
    bool prune_large;
};

// Control block: int[8] (count, next count, status, split-sampled, survivors,
// clones, kept splits, previous count) followed by two u64 Philox offsets.
constexpr size_t kDensityControlBytes = 8 * sizeof(int) + 2 * sizeof(unsigned long long);

struct DensityDecideArgs {
    const float* params;
    const float* sums;
    const float* abs_sums;
    const unsigned int* obs;
    int* control;
    int4* counts;       // [n + 1] (keep, clone, split sampled, split kept)
    int4* offsets;      // [n + 1] exclusive scan of counts
    int4* scan_scratch;  // density_scan_scratch_bytes(n)
    int* additions;     // [n + 1] (cap only)
    void* int_scan_scratch;  // scan_scratch_bytes(n) (cap only)
    int n;
    int max_count;      // 0 = no cap
    int random_blocks;
    DensityThresholds th;
    const int8_t* actions;  // optional learned proposals: 0 keep, 1 clone, 2 split, 3 prune, < 0 plain rule
};

struct DensityApplyArgs {
    const float* params;
    const int4* counts;
    const int4* offsets;
    int* control;
    float* samples;     // >= 6 * n floats
    float* out;         // 58 x out_stride
    int* history_parents;  // may be null
    int* parents;
    float* new_flags;
    float* sums;
    float* abs_sums;
    unsigned int* obs;
    int n;
    int out_stride;
    int random_blocks;
    unsigned long long seed;
    bool bf16_sh;       // precision-form layout (10 fp32 rows + 48 bf16 SH rows)
};

int launch_density_init(int* control, int count, cudaStream_t s);
int launch_density_accumulate(const float* stats, const float* abs_stats, const int* control, float* sums,
                              float* abs_sums, unsigned int* counts, int n, cudaStream_t s);
int launch_density_accumulate_observations(const float* grads, const float* radii, const int* ids, const int* control,
                                           float* sums, unsigned int* counts, int observations, cudaStream_t s);
size_t density_scan_scratch_bytes(int n);
int launch_density_decide(const DensityDecideArgs& a, cudaStream_t s);
int launch_density_prepare(const int4* offsets, int* control, int n, int random_blocks, cudaStream_t s);
int launch_density_apply(const DensityApplyArgs& a, cudaStream_t s);
// Decision codes of the last decide (0 keep, 1 clone, 2 split, 3 prune).
int launch_density_codes(const int4* counts, int n, int8_t* codes, cudaStream_t s);
// The 16 statistics of the learned density policy, [n][16] floats (density.cu).
// Per-Gaussian statistics the learned density policy adds to the round
// statistics (device arrays of the count; iteration = the current one).
struct LearnedStatsView {
    const float* max_radius;
    const float* depth_sum;
    const float* depth_sq;
    const float4* last_grad;
    const int* birth;
    int iteration;
};
// The 16 policy features per Gaussian ([n][16]); see density.cu.
int launch_density_features(const float* params, const float* sums, const unsigned int* obs, int n,
                            const DensityThresholds& th, float extent, const LearnedStatsView& ls, bool bf16_sh,
                            float* features, cudaStream_t s);
// birth[i] = prev_birth[history_parents[i]] where that is >= 0, else now.
int launch_birth_remap(const int* history_parents, const int* prev_birth, int prev_count, int* birth, int count,
                       int now, cudaStream_t s);
int launch_density_reset_opacity(const int* control, float* params, int stride, float max_logit, cudaStream_t s);

}  // namespace gsn
