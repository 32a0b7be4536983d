// Shared device-side definitions for the gs-native B200 kernels (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "gsn_types.h"
#include "profile.h"

namespace gsn {

constexpr int kTile = GSN_TILE_SIZE;           // 16x16 pixel tiles (renderer.cu:11)
constexpr int kTilePixels = kTile * kTile;
constexpr int kParams = GSN_PARAM_COUNT;       // 58 rows per Gaussian
constexpr int kShStride = GSN_SH_COEFFS;       // 16 coefficients per colour channel
constexpr float kLowPass = 0.3f;               // screen-space dilation (renderer.cu:12)
constexpr float kFovClamp = 1.3f;              // Jacobian clamp (renderer.cu:13)
constexpr float kNearFloor = 1e-6f;            // renderer.cu:14
constexpr float kAlphaMax = 0.99f;             // renderer.cu:315
constexpr float kAlphaMin = 1.0f / 255.0f;     // renderer.cu:316
constexpr float kTransmittanceMin = 1e-4f;     // renderer.cu:320

// Real spherical-harmonics normalisation constants, degrees 0-3 (standard values;
// same table as renderer.cu:17-30).
constexpr float kSh0 = 0.28209479177387814f;
constexpr float kSh1 = 0.4886025119029199f;
constexpr float kSh2a = 1.0925484305920792f;
constexpr float kSh2b = 0.31539156525252005f;
constexpr float kSh2c = 0.5462742152960396f;
constexpr float kSh3a = 0.5900435899266435f;
constexpr float kSh3b = 2.890611442640554f;
constexpr float kSh3c = 0.4570457994644658f;
constexpr float kSh3d = 0.3731763325901154f;
constexpr float kSh3e = 1.445305721320277f;

__host__ __device__ inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// Status helper: map the last launch error to a gsn status.
inline int launch_status() {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return GSN_OK;
    return e == cudaErrorMemoryAllocation ? GSN_ERR_OUT_OF_MEMORY : GSN_ERR_CUDA;
}

// Counts `kernels` launches of this library, then returns the launch status.
inline int launched(int kernels) {
    note_launch(kernels);
    return launch_status();
}

// ---------------------------------------------------------------- launches
// The training step's kernels are launched with programmatic stream
// serialization (sm_90 and later) on eager streams, so the next grid's CTAs are
// scheduled while the current grid drains instead of after it has retired. Each such kernel
// starts with pdl_begin(): it waits until its predecessor has completed and its
// memory is visible (griddepcontrol.wait, a no-op for a grid launched without
// the attribute), then lets its own dependents be scheduled
// (griddepcontrol.launch_dependents: they run once every CTA of this grid has
// started, and wait for it in turn). Nothing a kernel reads from an earlier
// launch is touched before pdl_begin().
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KernelArgs, typename... Args>
inline void launch_step(void (*kernel)(KernelArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                        Args&&... args) {
    cudaLaunchAttribute attribute[1];
    attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attribute[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t config{};
    config.gridDim = grid;
    config.blockDim = block;
    config.dynamicSmemBytes = smem;
    config.stream = stream;
    config.attrs = attribute;
    // eager streams only: inside a captured graph the launches already follow
    // each other without host latency, and programmatic edges measured slower
    // there (chosen form 780 -> 773 it/s; culled sparse form 751 -> 717)
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    const bool capturing = cudaStreamIsCapturing(stream, &capture) == cudaSuccess &&
                           capture != cudaStreamCaptureStatusNone;
    config.numAttrs = programmatic_launch() && !capturing ? 1 : 0;
    cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...);
}

// ---------------------------------------------------------------- layouts
// Parameter block layouts. The plain form uses the reference's 58 fp32 rows of
// stride N. The precision form keeps the 10 geometry rows (position, log-scale,
// axis-angle, opacity logit) in fp32 and stores the 48 SH coefficients in bf16
// as 24 pair rows right after them: pair row r holds coefficients 2r (low 16
// bits) and 2r + 1 (high 16 bits) of Gaussian i in the 32-bit word r * N + i,
// so its block is 10 + 24 = 34 rows of 32-bit words of stride N, and every SH
// load or store moves 4 bytes per Gaussian like an fp32 row. Adam's moments use
// the same layout as the parameters.
constexpr int kGeometryRows = GSN_SH_INDEX;  // 10
constexpr int kShRows = 3 * kShStride;       // 48
constexpr int kShPairRows = kShRows / 2;     // 24
constexpr int kPrecisionPhysicalRows = kGeometryRows + kShPairRows;  // 34

template <bool kBf16>
__host__ __device__ constexpr int physical_rows() { return kBf16 ? kPrecisionPhysicalRows : kParams; }

// bf16 bits <-> fp32 (bf16 is the upper half of an fp32: exact widening).
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

// SH coefficient k (0..47, channel-major) of Gaussian i.
template <bool kBf16>
__device__ __forceinline__ float load_sh(const float* block, int64_t n, int k, int64_t i) {
    if constexpr (kBf16) {
        const uint32_t w = reinterpret_cast<const uint32_t*>(block)[(kGeometryRows + (k >> 1)) * n + i];
        return (k & 1) ? bf16_hi(w) : bf16_lo(w);
    } else {
        return block[(kGeometryRows + k) * n + i];
    }
}

// The K coefficients k0 .. k0 + K - 1 (k0 even) of Gaussian i, one 32-bit load
// per pair in the precision layout.
template <bool kBf16, int K>
__device__ __forceinline__ void load_sh_coefs(const float* block, int64_t n, int k0, int64_t i, float* out) {
    if constexpr (kBf16) {
        const uint32_t* words = reinterpret_cast<const uint32_t*>(block);
#pragma unroll
        for (int q = 0; 2 * q < K; ++q) {
            const uint32_t w = words[(kGeometryRows + (k0 >> 1) + q) * n + i];
            out[2 * q] = bf16_lo(w);
            if (2 * q + 1 < K) out[2 * q + 1] = bf16_hi(w);
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = block[(kGeometryRows + k0 + k) * n + i];
    }
}

// 32-bit xorshift generator (Marsaglia 2003) for stochastic rounding; seeded per
// thread with the MurmurHash3 finaliser of (element, step).
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ uint32_t xorshift32(uint32_t& x) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return x;
}

// fp32 -> bf16 by stochastic rounding: the 16 dropped mantissa bits decide the
// direction with probability equal to their fraction of an ulp, so the rounding
// is unbiased and small Adam steps accumulate in expectation. Inf and NaN
// convert as with round-to-nearest.
__device__ __forceinline__ __nv_bfloat16 bf16_stochastic(float x, uint32_t noise16) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) == 0x7f800000u) return __float2bfloat16_rn(x);
    u += noise16 & 0xffffu;
    return __ushort_as_bfloat16(static_cast<unsigned short>(u >> 16));
}

// Rodrigues rotation of an axis-angle vector. The expression order is the one
// the reference uses in renderer.cu:35-66 and solver.cu:185-221, which the
// bit-exact parity of tile keys depends on.
__device__ __forceinline__ void axis_angle_to_matrix(float rx, float ry, float rz, float R[9]) {
    float angle = sqrtf(rx * rx + ry * ry + rz * rz);
    if (angle < 1e-8f) {
        R[0] = 1.0f; R[1] = 0.0f; R[2] = 0.0f;
        R[3] = 0.0f; R[4] = 1.0f; R[5] = 0.0f;
        R[6] = 0.0f; R[7] = 0.0f; R[8] = 1.0f;
        return;
    }
    float x = rx / angle;
    float y = ry / angle;
    float z = rz / angle;
    float c = cosf(angle);
    float s = sinf(angle);
    float t = 1.0f - c;
    R[0] = c + t * x * x;
    R[1] = t * x * y - s * z;
    R[2] = t * x * z + s * y;
    R[3] = t * x * y + s * z;
    R[4] = c + t * y * y;
    R[5] = t * y * z - s * x;
    R[6] = t * x * z - s * y;
    R[7] = t * y * z + s * x;
    R[8] = c + t * z * z;
}

}  // namespace gsn
