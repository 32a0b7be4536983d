// Spatial (Morton) ordering of the Gaussians and the gathers that apply it.
//
// A permutation of the Gaussians changes no result (every kernel is per
// Gaussian, per record or per pixel, and tile lists are ordered by depth, then
// id: reordering ids only changes which of two equal-depth Gaussians comes
// first, exactly as the reference's own ordering after a density step does).
// It does change locality: with the ids in Morton order of their means, the
// Gaussians of one view occupy long id runs, so a visibility-masked update
// (GaussianUpdateArgs::sparse) skips whole 32-byte sectors of the SoA rows, and
// the per-record gathers and gradient atomics of a tile hit nearby addresses.
//
// Keys: 10 bits per axis of the position inside the bounding box of all
// finite means (a device min/max reduction), interleaved z-y-x into 30 bits.
#include "common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

// Order-preserving float <-> int map for atomicMin / atomicMax.
__device__ __forceinline__ int ordered(float f) {
    const int b = __float_as_int(f);
    return b >= 0 ? b : b ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float unordered(int b) { return __int_as_float(b >= 0 ? b : b ^ 0x7FFFFFFF); }

__global__ void bounds_init(int* bounds) {
    const int t = threadIdx.x;
    if (t < 3) bounds[t] = 0x7FFFFFFF;
    else if (t < 6) bounds[t] = static_cast<int>(0x80000000u);
}

__global__ void __launch_bounds__(256) position_bounds(const float* __restrict__ params, int n,
                                                       int* __restrict__ bounds) {
    float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float x = params[static_cast<int64_t>(a) * n + i];
            if (isfinite(x)) {
                lo[a] = fminf(lo[a], x);
                hi[a] = fmaxf(hi[a], x);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            atomicMin(bounds + a, ordered(lo[a]));
            atomicMax(bounds + 3 + a, ordered(hi[a]));
        }
    }
}

__device__ __forceinline__ uint32_t spread10(uint32_t x) {
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__global__ void __launch_bounds__(256) morton_keys(const float* __restrict__ params, int n,
                                                   const int* __restrict__ bounds, uint32_t* __restrict__ keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float lo = unordered(bounds[a]), hi = unordered(bounds[3 + a]);
        const float x = params[static_cast<int64_t>(a) * n + i];
        const float span = hi - lo;
        float f = span > 0.0f ? (x - lo) / span : 0.0f;
        f = isfinite(f) ? fminf(fmaxf(f, 0.0f), 1.0f) : 1.0f;
        q[a] = static_cast<uint32_t>(f * 1023.0f + 0.5f);
    }
    keys[i] = spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
}

template <typename T>
__global__ void __launch_bounds__(256) gather_rows(const T* __restrict__ src, T* __restrict__ dst,
                                                   const uint32_t* __restrict__ perm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t row = static_cast<int64_t>(blockIdx.y) * n;
    dst[row + i] = src[row + perm[i]];
}

__global__ void __launch_bounds__(256) compose_parents(const int* __restrict__ parents,
                                                       const uint32_t* __restrict__ perm, int n,
                                                       int* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = static_cast<int>(perm[i]);
    out[i] = parents ? parents[p] : p;
}

}  // namespace

int launch_morton_keys(const float* params, int n, int* bounds, uint32_t* keys, cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    if (!params || !bounds || !keys) return GSN_ERR_INVALID_ARGUMENT;
    bounds_init<<<1, 32, 0, stream>>>(bounds);
    position_bounds<<<min(ceil_div(n, 256), 148 * 8), 256, 0, stream>>>(params, n, bounds);
    morton_keys<<<ceil_div(n, 256), 256, 0, stream>>>(params, n, bounds, keys);
    return launched(3);
}

int launch_gather_gaussians(const float* src, float* dst, const uint32_t* perm, int n, bool bf16_sh,
                            cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    if (!src || !dst || !perm) return GSN_ERR_INVALID_ARGUMENT;
    const unsigned blocks = static_cast<unsigned>(ceil_div(n, 256));
    // one 32-bit word per (physical row, Gaussian) in both layouts
    gather_rows<float><<<dim3(blocks, bf16_sh ? kPrecisionPhysicalRows : kParams), 256, 0, stream>>>(src, dst, perm, n);
    return launched(1);
}

int launch_compose_parents(const int* parents, const uint32_t* perm, int n, int* out, cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    if (!perm || !out) return GSN_ERR_INVALID_ARGUMENT;
    compose_parents<<<ceil_div(n, 256), 256, 0, stream>>>(parents, perm, n, out);
    return launched(1);
}

}  // namespace gsn
