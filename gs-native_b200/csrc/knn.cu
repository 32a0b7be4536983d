// (h) LBVH 3-nearest-neighbour search for the initial Gaussian scales.
//
// Same result as ComputeMeanDist2Cuda (knn.cu:16-255): for every point the mean
// of its (up to) three smallest squared distances to the other points, 0 when
// there are fewer than two points. The structure is a linear BVH: 30-bit Morton
// codes over the bounding box, a stable radix sort (sort.cu), buckets of 8
// consecutive sorted points as leaves, and an implicit complete binary tree of
// bucket boxes built bottom-up level by level. Each query walks the tree with an
// explicit stack, pruning nodes whose box is farther than the current third-best
// distance. Squared distances are evaluated without contraction
// ((dx*dx + dy*dy) + dz*dz, each rounded) and ties go to the smaller index, so the
// neighbour indices equal those of an exhaustive FP32 search.
#include <float.h>

#include "common.cuh"
#include "kernels.h"
#include "knn_kernels.h"

namespace gsn {

namespace {

constexpr int kThreads = 256;
constexpr int kBucket = 8;

__device__ __forceinline__ unsigned int spread10(unsigned int v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ unsigned int float_to_ordered(float f) {
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float ordered_to_float(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__global__ void bounds_kernel(const float* __restrict__ pts, int n, unsigned int* bounds) {
    __shared__ unsigned int s[6];
    if (threadIdx.x < 6) s[threadIdx.x] = threadIdx.x < 3 ? 0xFFFFFFFFu : 0u;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            unsigned int o = float_to_ordered(pts[3ll * i + a]);
            atomicMin(&s[a], o);
            atomicMax(&s[3 + a], o);
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(bounds + threadIdx.x, s[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(bounds + threadIdx.x, s[threadIdx.x]);
}

__global__ void morton_kernel(const float* __restrict__ pts, int n, const unsigned int* __restrict__ bounds,
                              uint32_t* __restrict__ keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float lo = ordered_to_float(bounds[a]), hi = ordered_to_float(bounds[3 + a]);
        float ext = hi - lo;
        float t = ext > 0.0f ? (pts[3ll * i + a] - lo) / ext : 0.0f;
        c[a] = static_cast<unsigned int>(fminf(fmaxf(t * 1023.0f, 0.0f), 1023.0f));
    }
    keys[i] = spread10(c[0]) | (spread10(c[1]) << 1) | (spread10(c[2]) << 2);
}

// Leaf boxes: bucket b covers sorted points [8b, 8b + 8).
__global__ void leaves_kernel(const float* __restrict__ pts, const uint32_t* __restrict__ order, int n, int leaves,
                              float4* __restrict__ lo, float4* __restrict__ hi) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= leaves) return;
    float3 mn = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), mx = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (int k = b * kBucket; k < min(n, (b + 1) * kBucket); ++k) {
        const float* p = pts + 3ll * order[k];
        mn = make_float3(fminf(mn.x, p[0]), fminf(mn.y, p[1]), fminf(mn.z, p[2]));
        mx = make_float3(fmaxf(mx.x, p[0]), fmaxf(mx.y, p[1]), fmaxf(mx.z, p[2]));
    }
    lo[leaves + b] = make_float4(mn.x, mn.y, mn.z, 0.0f);
    hi[leaves + b] = make_float4(mx.x, mx.y, mx.z, 0.0f);
}

__global__ void level_kernel(float4* __restrict__ lo, float4* __restrict__ hi, int begin) {
    const int node = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= 2 * begin) return;
    float4 a = lo[2 * node], b = lo[2 * node + 1];
    lo[node] = make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.0f);
    a = hi[2 * node];
    b = hi[2 * node + 1];
    hi[node] = make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), 0.0f);
}

__device__ __forceinline__ float box_distance(float3 p, float4 lo, float4 hi) {
    float x = fmaxf(fmaxf(lo.x - p.x, p.x - hi.x), 0.0f);
    float y = fmaxf(fmaxf(lo.y - p.y, p.y - hi.y), 0.0f);
    float z = fmaxf(fmaxf(lo.z - p.z, p.z - hi.z), 0.0f);
    return x * x + y * y + z * z;
}

// Exact squared distance in FP32 without contraction: ((dx*dx + dy*dy) + dz*dz).
__device__ __forceinline__ float sq_distance(float3 p, const float* q) {
    float dx = __fsub_rn(p.x, q[0]), dy = __fsub_rn(p.y, q[1]), dz = __fsub_rn(p.z, q[2]);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

struct Best3 {
    float d[3];
    int i[3];
    __device__ __forceinline__ void init() {
        d[0] = d[1] = d[2] = FLT_MAX;
        i[0] = i[1] = i[2] = -1;
    }
    __device__ __forceinline__ bool better(float dist, int idx, int k) const {
        return dist < d[k] || (dist == d[k] && (i[k] < 0 || idx < i[k]));
    }
    __device__ __forceinline__ void insert(float dist, int idx) {
        if (!better(dist, idx, 2)) return;
        if (better(dist, idx, 1)) {
            d[2] = d[1];
            i[2] = i[1];
            if (better(dist, idx, 0)) {
                d[1] = d[0];
                i[1] = i[0];
                d[0] = dist;
                i[0] = idx;
            } else {
                d[1] = dist;
                i[1] = idx;
            }
        } else {
            d[2] = dist;
            i[2] = idx;
        }
    }
};

__global__ void __launch_bounds__(kThreads) query_kernel(const float* __restrict__ pts,
                                                         const uint32_t* __restrict__ order, int n, int leaves,
                                                         const float4* __restrict__ lo, const float4* __restrict__ hi,
                                                         float* __restrict__ mean_dist2, int* __restrict__ neighbors,
                                                         int* __restrict__ status) {
    const int rank = blockIdx.x * blockDim.x + threadIdx.x;
    if (rank >= n) return;
    const int self = static_cast<int>(order[rank]);
    const float* sp = pts + 3ll * self;
    const float3 p = make_float3(sp[0], sp[1], sp[2]);
    Best3 best;
    best.init();
    int stack[64];
    int size = 0;
    int node = 1;
    // boxes are pruned against the current third distance widened by a few ulps,
    // so rounding of the box distance can never drop a tying candidate
    while (true) {
        if (box_distance(p, lo[node], hi[node]) <= best.d[2] * 1.000004f) {
            if (node >= leaves) {
                const int b = node - leaves;
                for (int k = b * kBucket; k < min(n, (b + 1) * kBucket); ++k) {
                    const int other = static_cast<int>(order[k]);
                    if (other == self) continue;
                    best.insert(sq_distance(p, pts + 3ll * other), other);
                }
            } else {
                const int left = 2 * node, right = left + 1;
                float dl = box_distance(p, lo[left], hi[left]);
                float dr = box_distance(p, lo[right], hi[right]);
                const int near = dl <= dr ? left : right, far = dl <= dr ? right : left;
                if (fmaxf(dl, dr) <= best.d[2] * 1.000004f) {
                    if (size < 64) {
                        stack[size++] = far;
                    } else {
                        atomicExch(status, 1);  // deeper than any tree this builds; report, do not overflow
                    }
                }
                node = near;
                continue;
            }
        }
        if (size == 0) break;
        node = stack[--size];
    }
    const int found = n - 1 < 3 ? n - 1 : 3;
    float mean = 0.0f;
    if (found == 3) mean = (best.d[0] + best.d[1] + best.d[2]) / 3.0f;
    else if (found == 2) mean = (best.d[0] + best.d[1]) / 2.0f;
    else if (found == 1) mean = best.d[0];
    mean_dist2[self] = mean;
    if (neighbors)
#pragma unroll
        for (int k = 0; k < 3; ++k) neighbors[3ll * self + k] = k < found ? best.i[k] : -1;
}

inline int grid_for(int64_t n) { return static_cast<int>(n > 0 ? (n + kThreads - 1) / kThreads : 1); }

}  // namespace

KnnLayout knn_layout(int n) {
    KnnLayout L;
    int buckets = (n + kBucket - 1) / kBucket;
    L.leaves = 1;
    while (L.leaves < buckets) L.leaves *= 2;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t at = off;
        off += (bytes + 255) & ~static_cast<size_t>(255);
        return at;
    };
    L.bounds = take(6 * sizeof(unsigned int));
    L.keys = take(sizeof(uint32_t) * static_cast<size_t>(n));
    L.keys_alt = take(sizeof(uint32_t) * static_cast<size_t>(n));
    L.ids = take(sizeof(uint32_t) * static_cast<size_t>(n));
    L.ids_alt = take(sizeof(uint32_t) * static_cast<size_t>(n));
    L.lo = take(sizeof(float4) * 2 * static_cast<size_t>(L.leaves));
    L.hi = take(sizeof(float4) * 2 * static_cast<size_t>(L.leaves));
    L.status = take(sizeof(int));
    L.sort = take(radix_sort_scratch_bytes(n));
    L.total = off;
    return L;
}

int launch_knn3(const float* points, int n, float* mean_dist2, int* neighbors, void* workspace, cudaStream_t s) {
    if (n <= 0) return GSN_OK;
    if (n < 2) {
        if (cudaMemsetAsync(mean_dist2, 0, sizeof(float) * n, s) != cudaSuccess) return GSN_ERR_CUDA;
        if (neighbors && cudaMemsetAsync(neighbors, 0xFF, sizeof(int) * 3 * n, s) != cudaSuccess) return GSN_ERR_CUDA;
        return GSN_OK;
    }
    const KnnLayout L = knn_layout(n);
    char* w = static_cast<char*>(workspace);
    auto* bounds = reinterpret_cast<unsigned int*>(w + L.bounds);
    auto* keys = reinterpret_cast<uint32_t*>(w + L.keys);
    auto* keys_alt = reinterpret_cast<uint32_t*>(w + L.keys_alt);
    auto* ids = reinterpret_cast<uint32_t*>(w + L.ids);
    auto* ids_alt = reinterpret_cast<uint32_t*>(w + L.ids_alt);
    auto* lo = reinterpret_cast<float4*>(w + L.lo);
    auto* hi = reinterpret_cast<float4*>(w + L.hi);
    auto* status = reinterpret_cast<int*>(w + L.status);
    const unsigned int init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
    if (cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess)
        return GSN_ERR_CUDA;
    bounds_kernel<<<grid_for(n), kThreads, 0, s>>>(points, n, bounds);
    morton_kernel<<<grid_for(n), kThreads, 0, s>>>(points, n, bounds, keys);
    int launches = 2;
    bool alt = false;
    RadixSortScratch scratch = radix_sort_scratch(w + L.sort, n);
    int st = launch_radix_sort(keys, ids, keys_alt, ids_alt, true, n, nullptr, 0, 30, scratch, &alt, s);
    if (st != GSN_OK) return st;
    const uint32_t* order = alt ? ids_alt : ids;
    leaves_kernel<<<grid_for(L.leaves), kThreads, 0, s>>>(points, order, n, L.leaves, lo, hi);
    ++launches;
    // padding leaves beyond the last bucket: empty boxes
    const int buckets = (n + kBucket - 1) / kBucket;
    for (int begin = L.leaves / 2; begin > 0; begin /= 2) {
        level_kernel<<<grid_for(begin), kThreads, 0, s>>>(lo, hi, begin);
        ++launches;
    }
    (void)buckets;
    query_kernel<<<grid_for(n), kThreads, 0, s>>>(points, order, n, L.leaves, lo, hi, mean_dist2, neighbors, status);
    ++launches;
    return launched(launches);
}

}  // namespace gsn
