// (e) Fused L1 + SSIM loss gradient w.r.t. the rendered image.
//
// L = 0.8 * mean|I - T| + 0.2 * (1 - mean SSIM(I, T)), 11x11 Gaussian window
// (sigma 1.5), zero padding, C1 = 1e-4, C2 = 9e-4. dL/dI is evaluated per pixel
// and channel in one pass: the five local moments are filtered separably, the
// per-centre SSIM partials (dSSIM/dmu, dSSIM/dE[xy], dSSIM/dE[x^2]) are formed,
// and filtered back with the same window (the window is symmetric, so the
// adjoint of the zero-padded filter is the filter itself). Every filter sum runs
// over its 11 taps in ascending order with the weights of solver.cu:14-24, which
// keeps the result bit-identical to the reference's kernel (solver.cu:26-168).
//
// Optionally the kernel also reduces the loss itself in FP64 (the reference
// never computes it): sum |I - T|, sum SSIM over the image's own centres and
// sum (I - T)^2 for the PSNR, accumulated with double atomics.
#include "common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

// Normalised 11-tap Gaussian, sigma 1.5 (the values of solver.cu:14-24).
__constant__ float c_window[11] = {1.028380120e-03f, 7.598758210e-03f, 3.600077330e-02f, 1.093606870e-01f,
                                   2.130055430e-01f, 2.660117150e-01f, 2.130055430e-01f, 1.093606870e-01f,
                                   3.600077330e-02f, 7.598758210e-03f, 1.028380120e-03f};

constexpr int kTw = 16;                // output tile width
constexpr int kTh = 32;                // output tile height
constexpr int kThreads = kTw * kTh;    // 512
constexpr int kInW = kTw + 20;         // raw input incl. 10-pixel halo
constexpr int kInH = kTh + 20;
constexpr int kMomW = kTw + 10;        // moment columns (centres incl. 5-pixel halo)
constexpr int kCenH = kTh + 10;        // centre rows
constexpr float kC1 = 0.0001f;
constexpr float kC2 = 0.0009f;

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w) s += red[w];
    return s;
}

__global__ void __launch_bounds__(kThreads, 3) loss_gradient_kernel(const float* __restrict__ image,
                                                                   const uint8_t* __restrict__ target,
                                                                   float* __restrict__ grad, int width, int height,
                                                                   double* __restrict__ sums) {
    // one arena, reused by the three stages
    __shared__ float s[5 * kInH * kMomW];
    __shared__ double red[kThreads / 32];
    const int t = threadIdx.x;
    const int ch = blockIdx.z;
    const int ox = blockIdx.x * kTw, oy = blockIdx.y * kTh;
    const int x = ox + t % kTw, y = oy + t / kTw;
    const bool inside = x < width && y < height;
    const int64_t pix = (static_cast<int64_t>(y) * width + x) * 3 + ch;
    const float I = inside ? image[pix] : 0.0f;
    const float R = inside ? target[pix] * (1.0f / 255.0f) : 0.0f;

    // stage 0: raw image / target with a 10-pixel zero-padded halo
    float* raw_i = s;
    float* raw_t = s + kInH * kInW;
    for (int j = t; j < kInH * kInW; j += kThreads) {
        int hx = ox + j % kInW - 10, hy = oy + j / kInW - 10;
        bool ok = hx >= 0 && hy >= 0 && hx < width && hy < height;
        int64_t k = (static_cast<int64_t>(hy) * width + hx) * 3 + ch;
        raw_i[j] = ok ? image[k] : 0.0f;
        raw_t[j] = ok ? target[k] * (1.0f / 255.0f) : 0.0f;
    }
    __syncthreads();

    // stage 1: horizontal filter of the five moments over kInH x kMomW
    constexpr int kHSlots = (kInH * kMomW + kThreads - 1) / kThreads;
    float h[kHSlots][5];
#pragma unroll
    for (int q = 0; q < kHSlots; ++q) {
#pragma unroll
        for (int m = 0; m < 5; ++m) h[q][m] = 0.0f;
        int j = t + q * kThreads;
        if (j < kInH * kMomW) {
            int base = (j / kMomW) * kInW + j % kMomW;
#pragma unroll
            for (int dx = 0; dx < 11; ++dx) {
                float w = c_window[dx];
                float a = raw_i[base + dx];
                float b = raw_t[base + dx];
                h[q][0] += w * a;
                h[q][1] += w * b;
                h[q][2] += w * a * a;
                h[q][3] += w * b * b;
                h[q][4] += w * a * b;
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kHSlots; ++q) {
        int j = t + q * kThreads;
        if (j < kInH * kMomW)
#pragma unroll
            for (int m = 0; m < 5; ++m) s[m * kInH * kMomW + j] = h[q][m];
    }
    __syncthreads();

    // stage 2: vertical filter -> moments at the kCenH x kMomW centres, then the
    // SSIM partials of every centre inside the image
    constexpr int kSSlots = (kCenH * kMomW + kThreads - 1) / kThreads;
    float mo[kSSlots][5];
#pragma unroll
    for (int q = 0; q < kSSlots; ++q) {
#pragma unroll
        for (int m = 0; m < 5; ++m) mo[q][m] = 0.0f;
        int j = t + q * kThreads;
        if (j < kCenH * kMomW) {
#pragma unroll
            for (int dy = 0; dy < 11; ++dy) {
                float w = c_window[dy];
                int k = (j / kMomW + dy) * kMomW + j % kMomW;
#pragma unroll
                for (int m = 0; m < 5; ++m) mo[q][m] += w * s[m * kInH * kMomW + k];
            }
        }
    }
    double ssim_sum = 0.0;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kSSlots; ++q) {
        int j = t + q * kThreads;
        if (j < kCenH * kMomW) {
            int cx = j % kMomW, cy = j / kMomW;
            int hx = ox + cx - 5, hy = oy + cy - 5;
            float pa = 0.0f, pb = 0.0f, pc = 0.0f;
            if (hx >= 0 && hy >= 0 && hx < width && hy < height) {
                float m = mo[q][0], n = mo[q][1];
                float inv_d = 1.0f / (m * m + n * n + kC1);
                float inv_e = 1.0f / (mo[q][2] - m * m + mo[q][3] - n * n + kC2);
                float lum = (2 * m * n + kC1) * inv_d;
                float cs = (2 * (mo[q][4] - m * n) + kC2) * inv_e;
                float dmu = 2 * (n - m * lum) * inv_d * cs;
                pb = 2 * lum * inv_e;
                pc = -lum * cs * inv_e;
                pa = dmu - n * pb - 2 * m * pc;
                if (sums && cx >= 5 && cx < 5 + kTw && cy >= 5 && cy < 5 + kTh)
                    ssim_sum += static_cast<double>(lum) * static_cast<double>(cs);
            }
            s[j] = pa;
            s[kCenH * kMomW + j] = pb;
            s[2 * kCenH * kMomW + j] = pc;
        }
    }
    __syncthreads();

    // stage 3: horizontal filter of the partials over kCenH x kTw
    constexpr int kGSlots = (kCenH * kTw + kThreads - 1) / kThreads;
    float g[kGSlots][3];
#pragma unroll
    for (int q = 0; q < kGSlots; ++q) {
        g[q][0] = g[q][1] = g[q][2] = 0.0f;
        int j = t + q * kThreads;
        if (j < kCenH * kTw) {
#pragma unroll
            for (int dx = 0; dx < 11; ++dx) {
                float w = c_window[dx];
                int k = (j / kTw) * kMomW + j % kTw + dx;
#pragma unroll
                for (int c = 0; c < 3; ++c) g[q][c] += w * s[c * kCenH * kMomW + k];
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kGSlots; ++q) {
        int j = t + q * kThreads;
        if (j < kCenH * kTw)
#pragma unroll
            for (int c = 0; c < 3; ++c) s[c * kCenH * kTw + j] = g[q][c];
    }
    __syncthreads();

    // stage 4: vertical filter at the output pixel and the combined gradient
    if (inside) {
        float f[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int dy = 0; dy < 11; ++dy) {
            float w = c_window[dy];
            int k = (t / kTw + dy) * kTw + t % kTw;
#pragma unroll
            for (int c = 0; c < 3; ++c) f[c] += w * s[c * kCenH * kTw + k];
        }
        float r = I - R;
        float l1 = static_cast<float>(r > 0) - static_cast<float>(r < 0);
        float dssim = -(f[0] + R * f[1] + 2 * I * f[2]);
        float norm = 1.0f / (3.0f * static_cast<float>(width) * height);
        grad[pix] = (0.8f * l1 + 0.2f * dssim) * norm;
    }
    if (sums) {
        double d = inside ? static_cast<double>(I) - static_cast<double>(R) : 0.0;
        double l1s = block_sum(fabs(d), red);
        double sq = block_sum(d * d, red);
        double ss = block_sum(ssim_sum, red);
        if (t == 0) {
            atomicAdd(sums + 0, l1s);
            atomicAdd(sums + 1, ss);
            atomicAdd(sums + 2, sq);
        }
    }
}

__global__ void finalize_loss_kernel(const double* sums, int width, int height, double* out) {
    double count = 3.0 * static_cast<double>(width) * height;
    double l1 = sums[0] / count, ssim = sums[1] / count, mse = sums[2] / count;
    out[0] = 0.8 * l1 + 0.2 * (1.0 - ssim);
    out[1] = l1;
    out[2] = ssim;
    out[3] = mse > 0.0 ? -10.0 * log10(mse) : INFINITY;
}

}  // namespace

int launch_loss_gradient(const float* image, const uint8_t* target, float* grad, int width, int height,
                         double* sums, cudaStream_t stream) {
    if (width <= 0 || height <= 0) return GSN_ERR_INVALID_ARGUMENT;
    if (sums && cudaMemsetAsync(sums, 0, 3 * sizeof(double), stream) != cudaSuccess) return GSN_ERR_CUDA;
    dim3 grid(ceil_div(width, kTw), ceil_div(height, kTh), 3);
    loss_gradient_kernel<<<grid, kThreads, 0, stream>>>(image, target, grad, width, height, sums);
    return launched(1);
}

int launch_finalize_loss(const double* sums, int width, int height, double* out, cudaStream_t stream) {
    finalize_loss_kernel<<<1, 1, 0, stream>>>(sums, width, height, out);
    return launched(1);
}

}  // namespace gsn
