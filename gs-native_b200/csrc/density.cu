// (g) Density control: clone / split / prune decision, four-way compaction
// offsets, Philox normal samples, child writing and statistics reset.
//
// Follows DensityController (density_controller.cu:26-647): the decision rules
// (60-116), the output order survivors | clones | first split children | second
// split children (219-221), the int4 compaction offsets (485-524), the control
// block with its Philox offset bookkeeping (118-136) and the child placement
// pos + R (n * s), log(s / 1.6) (168-243). Normal samples come from the same
// curand Philox4_32_10 stream with the same (seed, subsequence, offset) scheme
// (138-166), so for identical inputs the new Gaussians are bit-identical.
//
// Addition over the reference: an optional cap on the Gaussian count. Clones and
// kept splits (each adds one Gaussian) are then accepted in id order while the
// new count stays within the cap; the others revert to plain survivors.
#include <curand_kernel.h>

#include "common.cuh"
#include "density.h"

namespace gsn {

namespace {

constexpr int kThreads = 256;

__global__ void density_init_kernel(int* control, int count) {
    for (int i = 0; i < 8; ++i) control[i] = 0;
    control[0] = count;
    control[1] = count;
    auto* offsets = reinterpret_cast<unsigned long long*>(control + 8);
    offsets[0] = 0;
    offsets[1] = 0;
}

__global__ void accumulate_round_kernel(const float* __restrict__ stats, const float* __restrict__ abs_stats,
                                        const int* __restrict__ control, float* __restrict__ sums,
                                        float* __restrict__ abs_sums, unsigned int* __restrict__ counts, int n) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n || id >= control[0]) return;
    sums[id] += stats[id];
    abs_sums[id] += abs_stats[id];
    counts[id] += static_cast<unsigned int>(stats[n + id]);
}

__global__ void accumulate_observations_kernel(const float* __restrict__ grads, const float* __restrict__ radii,
                                               const int* __restrict__ ids, const int* __restrict__ control,
                                               float* __restrict__ sums, unsigned int* __restrict__ counts,
                                               int observations) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= observations || !(radii[k] > 0)) return;
    const int id = ids ? ids[k] : k;
    if (id < 0 || id >= control[0]) return;
    float x = grads[2ll * k], y = grads[2ll * k + 1];
    atomicAdd(sums + id, sqrtf(x * x + y * y));
    atomicAdd(counts + id, 1u);
}

// The plain threshold rule for one Gaussian (density_controller.cu:60-116):
// (survive, clone, split sampled, split kept).
__device__ __forceinline__ int4 plain_decision(const float* __restrict__ params, const float* __restrict__ sums,
                                               const float* __restrict__ abs_sums, const unsigned int* __restrict__ obs,
                                               int64_t N, int id, const DensityThresholds& th) {
    float opacity = 1.0f / (1.0f + expf(-params[static_cast<int64_t>(GSN_OPACITY_INDEX) * N + id]));
    float gradient = obs[id] ? sums[id] / obs[id] : 0;
    if (isnan(gradient)) gradient = 0;
    float s[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) s[a] = expf(params[static_cast<int64_t>(GSN_LOG_SCALE_INDEX + a) * N + id]);
    float max_scale = fmaxf(s[0], fmaxf(s[1], s[2]));
    if (isnan(s[0]) || isnan(s[1]) || isnan(s[2])) max_scale = nanf("");
    bool selected = gradient >= th.gradient_threshold;
    bool clone = selected && max_scale <= th.split_threshold;
    float abs_gradient = obs[id] ? abs_sums[id] / obs[id] : 0;
    bool split_selected =
        th.absolute_gradient_threshold > 0.0f ? abs_gradient >= th.absolute_gradient_threshold : selected;
    bool split = split_selected && max_scale > th.split_threshold;
    float remaining = max_scale;
    if (split && th.prune_large) {
        float x = expf(logf(s[0] / 1.6f));
        float y = expf(logf(s[1] / 1.6f));
        float z = expf(logf(s[2] / 1.6f));
        remaining = fmaxf(x, fmaxf(y, z));
        if (isnan(x) || isnan(y) || isnan(z)) remaining = nanf("");
    }
    bool remove = opacity < th.min_opacity || (th.prune_large && remaining > th.max_world_size);
    return make_int4(!split && !remove, clone && !remove, split, split && !remove);
}

// Decision of an action code (learned policy): 0 keep, 1 clone, 2 split, 3 prune.
__device__ __forceinline__ int4 action_decision(int action) {
    switch (action) {
        case 1: return make_int4(1, 1, 0, 0);
        case 2: return make_int4(0, 0, 1, 1);
        case 3: return make_int4(0, 0, 0, 0);
        default: return make_int4(1, 0, 0, 0);
    }
}

__global__ void decide_kernel(const float* __restrict__ params, const float* __restrict__ sums,
                              const float* __restrict__ abs_sums, const unsigned int* __restrict__ obs,
                              const int* __restrict__ control, const int8_t* __restrict__ actions,
                              int4* __restrict__ counts, int* __restrict__ additions, int n, DensityThresholds th) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id > n) return;
    if (id == n || id >= control[0]) {
        counts[id] = make_int4(0, 0, 0, 0);
        if (additions && id < n) additions[id] = 0;
        return;
    }
    int4 c = plain_decision(params, sums, abs_sums, obs, n, id, th);
    // a learned proposal replaces the plain decision where one is given (>= 0)
    if (actions && actions[id] >= 0) c = action_decision(actions[id]);
    counts[id] = c;
    if (additions) additions[id] = c.y || c.w ? 1 : 0;
}

__global__ void codes_kernel(const int4* __restrict__ counts, int n, int8_t* __restrict__ codes) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const int4 c = counts[id];
    codes[id] = c.z ? 2 : (c.y ? 1 : (c.x ? 0 : 3));
}

// The 16 per-Gaussian statistics of the learned density policy, the list the
// policy is specified on (accumulated view-space gradient norm and count, max
// screen radius, 3 log-scales, opacity, SH DC norm and higher-band energy,
// depth mean / variance, age, last-step gradient norms of mean / scale /
// opacity / SH), each scaled to order one:
//  0 round mean view-space gradient / gradient threshold   1 log(1 + round observations)
//  2 log(1 + round max screen radius, px)                  3-5 log-scale - log(split threshold)
//  6 opacity                                               7 |SH DC|
//  8 higher-band SH energy (sum of squares)                9 round mean depth / scene extent
// 10 round depth variance / extent^2                       11 age / 1000 iterations
// 12-15 log(1 + 1e4 |g|) of the last visible step's gradient of mean, log-scale, opacity logit, SH
template <bool kBf16>
__global__ void features_kernel(const float* __restrict__ params, const float* __restrict__ sums,
                                const unsigned int* __restrict__ obs, int n, DensityThresholds th, float extent,
                                LearnedStatsView ls, float* __restrict__ out) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const int64_t N = n;
    const float count = static_cast<float>(obs[id]);
    const float logit = params[static_cast<int64_t>(GSN_OPACITY_INDEX) * N + id];
    const float lsplit = logf(fmaxf(th.split_threshold, 1e-12f));
    float dc = 0.0f, rest = 0.0f;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float d = load_sh<kBf16>(params, N, ch * kShStride, id);
        dc += d * d;
#pragma unroll
        for (int k = 1; k < kShStride; ++k) {
            const float v = load_sh<kBf16>(params, N, ch * kShStride + k, id);
            rest += v * v;
        }
    }
    const float e = fmaxf(extent, 1e-12f);
    const float dmean = count > 0.0f ? ls.depth_sum[id] / count : 0.0f;
    const float dvar = count > 0.0f ? fmaxf(ls.depth_sq[id] / count - dmean * dmean, 0.0f) : 0.0f;
    const float4 g = ls.last_grad[id];
    float f[16];
    f[0] = fminf(count > 0.0f ? sums[id] / count / th.gradient_threshold : 0.0f, 50.0f);
    f[1] = log1pf(count);
    f[2] = log1pf(fmaxf(ls.max_radius[id], 0.0f));
#pragma unroll
    for (int a = 0; a < 3; ++a)
        f[3 + a] = fminf(fmaxf(params[static_cast<int64_t>(GSN_LOG_SCALE_INDEX + a) * N + id] - lsplit, -10.0f), 10.0f);
    f[6] = 1.0f / (1.0f + expf(-logit));
    f[7] = sqrtf(dc);
    f[8] = fminf(rest, 50.0f);
    f[9] = fminf(dmean / e, 50.0f);
    f[10] = fminf(dvar / (e * e), 50.0f);
    f[11] = fminf(static_cast<float>(max(ls.iteration - ls.birth[id], 0)) * 1e-3f, 50.0f);
    f[12] = log1pf(1e4f * g.x);
    f[13] = log1pf(1e4f * g.y);
    f[14] = log1pf(1e4f * g.z);
    f[15] = log1pf(1e4f * g.w);
#pragma unroll
    for (int k = 0; k < 16; ++k)
        if (!isfinite(f[k])) f[k] = 0.0f;
    float4* o = reinterpret_cast<float4*>(out + static_cast<int64_t>(id) * 16);
    o[0] = make_float4(f[0], f[1], f[2], f[3]);
    o[1] = make_float4(f[4], f[5], f[6], f[7]);
    o[2] = make_float4(f[8], f[9], f[10], f[11]);
    o[3] = make_float4(f[12], f[13], f[14], f[15]);
}

// Birth iteration after a density step: a Gaussian that keeps an old index's
// history (history_parents >= 0) keeps that Gaussian's birth; clones and split
// children are born now.
__global__ void birth_remap_kernel(const int* __restrict__ history_parents, const int* __restrict__ prev_birth,
                                   int prev_count, int* __restrict__ birth, int count, int now) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= count) return;
    const int p = history_parents ? history_parents[id] : -1;
    birth[id] = p >= 0 && p < prev_count ? prev_birth[p] : now;
}

// Cap: accept additions (clone or kept split) in id order while the count stays
// within max_count; base = survivors + kept-split parents (totals of the first scan).
__global__ void cap_kernel(int4* __restrict__ counts, const int* __restrict__ addition_prefix,
                           const int4* __restrict__ totals, int n, int max_count) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    int4 c = counts[id];
    bool adds = c.y || c.w;
    if (!adds) return;
    const int base = totals->x + totals->w;
    const int budget = max(0, max_count - base);
    if (addition_prefix[id] < budget) return;
    if (c.w) c = make_int4(1, 0, 0, 0);  // the split parent survives unchanged
    else c.y = 0;                           // no clone
    counts[id] = c;
}

// ---------------------------------------------------------------- int4 scan
constexpr int kScanItems = 8;
constexpr int kScanChunk = kThreads * kScanItems;

__device__ __forceinline__ int4 add4(int4 a, int4 b) { return make_int4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }

__device__ __forceinline__ int4 shfl_up4(int4 v, int o) {
    return make_int4(__shfl_up_sync(0xffffffffu, v.x, o), __shfl_up_sync(0xffffffffu, v.y, o),
                     __shfl_up_sync(0xffffffffu, v.z, o), __shfl_up_sync(0xffffffffu, v.w, o));
}

__device__ __forceinline__ int4 block_exclusive4(int4 x, int4* warp_sums, int4* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int4 inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int4 y = shfl_up4(inc, o);
        if (lane >= o) inc = add4(inc, y);
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    int4 prefix = make_int4(0, 0, 0, 0), sum = make_int4(0, 0, 0, 0);
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        int4 s = warp_sums[w];
        if (w < warp) prefix = add4(prefix, s);
        sum = add4(sum, s);
    }
    __syncthreads();
    *total = sum;
    int4 ex = add4(prefix, inc);
    return make_int4(ex.x - x.x, ex.y - x.y, ex.z - x.z, ex.w - x.w);
}

__global__ void scan4_reduce(const int4* __restrict__ in, int n, int4* __restrict__ block_sums) {
    __shared__ int4 warp_sums[kThreads / 32];
    const int64_t start = static_cast<int64_t>(blockIdx.x) * kScanChunk;
    int4 s = make_int4(0, 0, 0, 0);
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = start + k * kThreads + threadIdx.x;
        if (i < n) s = add4(s, in[i]);
    }
    int4 total;
    block_exclusive4(s, warp_sums, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void scan4_blocks(int4* __restrict__ block_sums, int blocks) {
    __shared__ int4 warp_sums[kThreads / 32];
    int4 carry = make_int4(0, 0, 0, 0);
    for (int base = 0; base < blocks; base += kThreads) {
        int i = base + threadIdx.x;
        int4 x = i < blocks ? block_sums[i] : make_int4(0, 0, 0, 0);
        int4 total;
        int4 ex = block_exclusive4(x, warp_sums, &total);
        if (i < blocks) block_sums[i] = add4(carry, ex);
        carry = add4(carry, total);
    }
}

__global__ void scan4_downsweep(const int4* __restrict__ in, int n, const int4* __restrict__ block_sums,
                                int4* __restrict__ out) {
    __shared__ int4 warp_sums[kThreads / 32];
    const int64_t start = static_cast<int64_t>(blockIdx.x) * kScanChunk + static_cast<int64_t>(threadIdx.x) * kScanItems;
    int4 v[kScanItems];
    int4 s = make_int4(0, 0, 0, 0);
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = start + k;
        v[k] = i < n ? in[i] : make_int4(0, 0, 0, 0);
        s = add4(s, v[k]);
    }
    int4 total;
    int4 run = add4(block_exclusive4(s, warp_sums, &total), block_sums[blockIdx.x]);
    for (int k = 0; k < kScanItems; ++k) {
        int64_t i = start + k;
        if (i < n) out[i] = run;
        run = add4(run, v[k]);
    }
}

// density_controller.cu:118-136: totals into the control block and the Philox
// offset advance of this round.
__global__ void prepare_kernel(const int4* __restrict__ offsets, int* control, int n, int random_blocks) {
    int4 totals = offsets[n];
    control[7] = control[0];
    control[1] = totals.x + totals.y + 2 * totals.w;
    control[2] = 0;
    control[3] = totals.z;
    control[4] = totals.x;
    control[5] = totals.y;
    control[6] = totals.w;
    auto* off = reinterpret_cast<unsigned long long*>(control + 8);
    unsigned long long numel = 6ull * totals.z;
    unsigned long long threads =
        min(static_cast<unsigned long long>(random_blocks), (numel + kThreads - 1) / kThreads) * kThreads;
    off[1] = off[0] + (numel ? ((numel - 1) / (4ull * threads) + 1) * 4ull : 0ull);
}

// density_controller.cu:138-166: 6 normal samples per split-selected Gaussian;
// thread k of `threads` owns subsequence k and writes slots k, k + threads, ...
__global__ void samples_kernel(const int* __restrict__ control, float* __restrict__ samples, int random_blocks,
                               unsigned long long seed) {
    const int64_t numel = 6ll * control[3];
    if (numel == 0) return;
    const int blocks = static_cast<int>(min(static_cast<int64_t>(random_blocks), (numel + kThreads - 1) / kThreads));
    if (static_cast<int>(blockIdx.x) >= blocks) return;
    const int64_t threads = static_cast<int64_t>(blocks) * kThreads;
    const int64_t index = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const int64_t rounded = ((numel - 1) / (4 * threads) + 1) * 4 * threads;
    const auto* off = reinterpret_cast<const unsigned long long*>(control + 8);
    curandStatePhilox4_32_10_t state;
    curand_init(seed, static_cast<unsigned long long>(index), off[0], &state);
    for (int64_t base = index; base < rounded; base += 4 * threads) {
        float4 values = curand_normal4(&state);
        const float v[4] = {values.x, values.y, values.z, values.w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            int64_t dst = base + c * threads;
            if (dst < numel) samples[dst] = v[c];
        }
    }
}

// density_controller.cu:168-243 (children) and 245-278 (parent ids, new flags,
// statistics reset), fused: one thread per source Gaussian. kBf16: precision-form
// layout (34 physical rows).
template <bool kBf16>
__global__ void write_kernel(const float* __restrict__ params, const int4* __restrict__ counts,
                             const int4* __restrict__ offsets, const int* __restrict__ control,
                             const float* __restrict__ samples, float* __restrict__ out,
                             int* __restrict__ history_parents, int* __restrict__ parents, float* __restrict__ new_flags,
                             int n, int out_stride) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= control[0]) return;
    const int64_t N = n;
    const int4 c = counts[id], o = offsets[id];
    const bool split = c.w != 0;
    if (!c.x && !c.y && !split) return;
    float scale[3] = {0.f, 0.f, 0.f}, R[9];
    if (split) {
#pragma unroll
        for (int a = 0; a < 3; ++a) scale[a] = expf(params[static_cast<int64_t>(GSN_LOG_SCALE_INDEX + a) * N + id]);
        float x = params[static_cast<int64_t>(GSN_ROTATION_INDEX) * N + id];
        float y = params[static_cast<int64_t>(GSN_ROTATION_INDEX + 1) * N + id];
        float z = params[static_cast<int64_t>(GSN_ROTATION_INDEX + 2) * N + id];
        float angle = sqrtf(x * x + y * y + z * z);
        float ca = 1.0f, cb = 0.5f;
        if (angle > 1e-4f) {
            ca = sinf(angle) / angle;
            float hs = sinf(angle * 0.5f) / (angle * 0.5f);
            cb = hs * hs * 0.5f;
        } else {
            float sq = angle * angle;
            ca -= sq / 6.0f;
            cb -= sq / 24.0f;
        }
        R[0] = 1 - cb * (y * y + z * z);
        R[1] = cb * x * y - ca * z;
        R[2] = cb * x * z + ca * y;
        R[3] = cb * x * y + ca * z;
        R[4] = 1 - cb * (x * x + z * z);
        R[5] = cb * y * z - ca * x;
        R[6] = cb * x * z - ca * y;
        R[7] = cb * y * z + ca * x;
        R[8] = 1 - cb * (x * x + y * y);
    }
    const int survivors = control[4], clones = control[5], kept_splits = control[6], sampled = control[3];
    const int children = split ? 2 : c.x + c.y;
    for (int child = 0; child < children; ++child) {
        const int dst = split ? survivors + clones + child * kept_splits + o.w
                              : (child == 0 && c.x ? o.x : survivors + o.y);
        // consistency guard: offsets that do not fit the output block mean the
        // decision buffers are stale; record it in the status word, write nothing
        if (dst < 0 || dst >= out_stride || (split && o.z >= sampled)) {
            atomicExch(const_cast<int*>(control) + 2, 1);
            return;
        }
        // every physical row is one 32-bit word per Gaussian; the SH rows (bf16
        // pairs in the precision layout) are copied bit for bit
        for (int p = 0; p < physical_rows<kBf16>(); ++p) {
            float value = params[static_cast<int64_t>(p) * N + id];
            if (split && p < GSN_POSITION_INDEX + 3) {
                float delta = 0;
                for (int a = 0; a < 3; ++a) {
                    int64_t k = (static_cast<int64_t>(child) * sampled + o.z) * 3 + a;
                    float local = samples[k] * scale[a];
                    delta += R[p * 3 + a] * local;
                }
                value += delta;
            } else if (split && p >= GSN_LOG_SCALE_INDEX && p < GSN_LOG_SCALE_INDEX + 3) {
                value = logf(scale[p - GSN_LOG_SCALE_INDEX] / 1.6f);
            }
            out[static_cast<int64_t>(p) * out_stride + dst] = value;
        }
        if (history_parents) history_parents[dst] = !split && child == 0 && c.x ? id : -1;
        parents[dst] = id;
        new_flags[dst] = c.y || c.z ? 1.0f : 0.0f;
    }
}

__global__ void finish_kernel(float* __restrict__ sums, float* __restrict__ abs_sums, unsigned int* __restrict__ obs,
                              int* control) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id < __ldg(control + 7)) {
        sums[id] = 0;
        abs_sums[id] = 0;
        obs[id] = 0;
    }
    if (id == 0) {
        control[0] = control[1];
        auto* off = reinterpret_cast<unsigned long long*>(control + 8);
        off[0] = off[1];
    }
}

__global__ void reset_opacity_kernel(const int* __restrict__ control, float* __restrict__ params, int stride,
                                     float max_logit) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= control[0]) return;
    const int64_t k = static_cast<int64_t>(GSN_OPACITY_INDEX) * stride + id;
    params[k] = fminf(params[k], max_logit);
}

inline int grid_for(int64_t n) { return static_cast<int>(n > 0 ? (n + kThreads - 1) / kThreads : 1); }

}  // namespace

int launch_density_init(int* control, int count, cudaStream_t s) {
    density_init_kernel<<<1, 1, 0, s>>>(control, count);
    return launched(1);
}

int launch_density_accumulate(const float* stats, const float* abs_stats, const int* control, float* sums,
                              float* abs_sums, unsigned int* counts, int n, cudaStream_t s) {
    if (n <= 0) return GSN_OK;
    accumulate_round_kernel<<<grid_for(n), kThreads, 0, s>>>(stats, abs_stats, control, sums, abs_sums, counts, n);
    return launched(1);
}

int launch_density_accumulate_observations(const float* grads, const float* radii, const int* ids, const int* control,
                                           float* sums, unsigned int* counts, int observations, cudaStream_t s) {
    if (observations <= 0) return GSN_OK;
    accumulate_observations_kernel<<<grid_for(observations), kThreads, 0, s>>>(grads, radii, ids, control, sums,
                                                                              counts, observations);
    return launched(1);
}

size_t density_scan_scratch_bytes(int n) {
    return (static_cast<size_t>((n + 1 + kScanChunk - 1) / kScanChunk) + 1) * sizeof(int4);
}

int launch_density_decide(const DensityDecideArgs& a, cudaStream_t s) {
    const int n = a.n;
    decide_kernel<<<grid_for(n + 1), kThreads, 0, s>>>(a.params, a.sums, a.abs_sums, a.obs, a.control, a.actions,
                                                      a.counts, a.max_count > 0 ? a.additions : nullptr, n, a.th);
    int launches = 1;
    const int blocks = (n + 1 + kScanChunk - 1) / kScanChunk;
    auto scan4 = [&]() {
        scan4_reduce<<<blocks, kThreads, 0, s>>>(a.counts, n + 1, a.scan_scratch);
        scan4_blocks<<<1, kThreads, 0, s>>>(a.scan_scratch, blocks);
        scan4_downsweep<<<blocks, kThreads, 0, s>>>(a.counts, n + 1, a.scan_scratch, a.offsets);
        launches += 3;
    };
    scan4();
    if (a.max_count > 0 && n > 0) {
        int st = launch_exclusive_scan(a.additions, nullptr, a.additions, n, a.int_scan_scratch, s);
        if (st != GSN_OK) return st;
        cap_kernel<<<grid_for(n), kThreads, 0, s>>>(a.counts, a.additions, a.offsets + n, n, a.max_count);
        launches += 1;
        scan4();
    }
    prepare_kernel<<<1, 1, 0, s>>>(a.offsets, a.control, n, a.random_blocks);
    return launched(launches + 1);
}

int launch_density_codes(const int4* counts, int n, int8_t* codes, cudaStream_t s) {
    if (n <= 0) return GSN_OK;
    codes_kernel<<<grid_for(n), kThreads, 0, s>>>(counts, n, codes);
    return launched(1);
}

int launch_density_features(const float* params, const float* sums, const unsigned int* obs, int n,
                            const DensityThresholds& th, float extent, const LearnedStatsView& ls, bool bf16_sh,
                            float* features, cudaStream_t s) {
    if (n <= 0) return GSN_OK;
    if (!ls.max_radius || !ls.depth_sum || !ls.depth_sq || !ls.last_grad || !ls.birth || !features)
        return GSN_ERR_INVALID_ARGUMENT;
    if (bf16_sh)
        features_kernel<true><<<grid_for(n), kThreads, 0, s>>>(params, sums, obs, n, th, extent, ls, features);
    else
        features_kernel<false><<<grid_for(n), kThreads, 0, s>>>(params, sums, obs, n, th, extent, ls, features);
    return launched(1);
}

int launch_birth_remap(const int* history_parents, const int* prev_birth, int prev_count, int* birth, int count,
                       int now, cudaStream_t s) {
    if (count <= 0) return GSN_OK;
    if (!birth || (prev_count > 0 && !prev_birth)) return GSN_ERR_INVALID_ARGUMENT;
    birth_remap_kernel<<<grid_for(count), kThreads, 0, s>>>(history_parents, prev_birth, prev_count, birth, count,
                                                           now);
    return launched(1);
}

int launch_density_prepare(const int4* offsets, int* control, int n, int random_blocks, cudaStream_t s) {
    prepare_kernel<<<1, 1, 0, s>>>(offsets, control, n, random_blocks);
    return launched(1);
}

int launch_density_apply(const DensityApplyArgs& a, cudaStream_t s) {
    samples_kernel<<<a.random_blocks, kThreads, 0, s>>>(a.control, a.samples, a.random_blocks, a.seed);
    if (a.bf16_sh)
        write_kernel<true><<<grid_for(a.n), kThreads, 0, s>>>(a.params, a.counts, a.offsets, a.control, a.samples,
                                                              a.out, a.history_parents, a.parents, a.new_flags, a.n,
                                                              a.out_stride);
    else
        write_kernel<false><<<grid_for(a.n), kThreads, 0, s>>>(a.params, a.counts, a.offsets, a.control, a.samples,
                                                               a.out, a.history_parents, a.parents, a.new_flags, a.n,
                                                               a.out_stride);
    finish_kernel<<<grid_for(a.n), kThreads, 0, s>>>(a.sums, a.abs_sums, a.obs, a.control);
    return launched(3);
}

int launch_density_reset_opacity(const int* control, float* params, int stride, float max_logit, cudaStream_t s) {
    if (stride <= 0) return GSN_OK;
    reset_opacity_kernel<<<grid_for(stride), kThreads, 0, s>>>(control, params, stride, max_logit);
    return launched(1);
}

}  // namespace gsn
