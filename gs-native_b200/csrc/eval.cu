// FP64 evaluation metrics of a rendered view against its u8 target, as the
// reference defines them for held-out views: RGB clamped to [0, 1], PSNR of
// the RGB mean squared error, SSIM with the 11 x 11 Gaussian window (sigma 1.5,
// zero padding, C1 = 1e-4, C2 = 9e-4 as the training loss), mean L1.
//
// One CTA per 32 x 8 pixel tile: the clamped image and the target of the
// 42 x 18 halo patch are staged in shared memory as doubles, the horizontal
// 11-tap pass writes the five moments (mu_x, mu_y, xx, yy, xy) of the 18 patch
// rows, and the vertical pass finishes SSIM per output pixel. Per-CTA sums go
// to a partials array that a single CTA reduces in a fixed order, so the
// result is deterministic. Off the training path (evaluation only).
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

constexpr int kTileX = 32, kTileY = 8, kRadius = 5, kTaps = 11;
constexpr int kPatchX = kTileX + 2 * kRadius, kPatchY = kTileY + 2 * kRadius;
constexpr int kEvalThreads = kTileX * kTileY;
constexpr int kReduceThreads = 512;

struct Window {
    double w[kTaps];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kEvalThreads) eval_metrics_kernel(const float* __restrict__ image,
                                                                    const uint8_t* __restrict__ target, int width,
                                                                    int height, Window win,
                                                                    double* __restrict__ partials) {
    __shared__ double a[kPatchY][kPatchX], b[kPatchY][kPatchX];
    __shared__ double h[5][kPatchY][kTileX];
    __shared__ double red[3][kEvalThreads / 32];
    const int tx = threadIdx.x, ty = threadIdx.y, t = ty * kTileX + tx;
    const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY;
    const int px = x0 + tx, py = y0 + ty;
    const bool inside = px < width && py < height;
    double ssim = 0.0, l1 = 0.0, sq = 0.0;
    for (int c = 0; c < 3; ++c) {
        for (int i = t; i < kPatchY * kPatchX; i += kEvalThreads) {
            const int r = i / kPatchX, q = i % kPatchX;
            const int gy = y0 - kRadius + r, gx = x0 - kRadius + q;
            double va = 0.0, vb = 0.0;
            if (gx >= 0 && gx < width && gy >= 0 && gy < height) {
                const size_t k = (static_cast<size_t>(gy) * width + gx) * 3 + c;
                va = fmin(fmax(static_cast<double>(image[k]), 0.0), 1.0);
                vb = target[k] / 255.0;
            }
            a[r][q] = va;
            b[r][q] = vb;
        }
        __syncthreads();
        for (int i = t; i < kPatchY * kTileX; i += kEvalThreads) {
            const int r = i / kTileX, q = i % kTileX;
            double m[5] = {0, 0, 0, 0, 0};
#pragma unroll
            for (int k = 0; k < kTaps; ++k) {
                const double va = a[r][q + k], vb = b[r][q + k], w = win.w[k];
                m[0] += w * va;
                m[1] += w * vb;
                m[2] += w * va * va;
                m[3] += w * vb * vb;
                m[4] += w * va * vb;
            }
#pragma unroll
            for (int j = 0; j < 5; ++j) h[j][r][q] = m[j];
        }
        __syncthreads();
        if (inside) {
            double m[5] = {0, 0, 0, 0, 0};
#pragma unroll
            for (int k = 0; k < kTaps; ++k)
#pragma unroll
                for (int j = 0; j < 5; ++j) m[j] += win.w[k] * h[j][ty + k][tx];
            const double ma = m[0], mb = m[1];
            const double va = m[2] - ma * ma, vb = m[3] - mb * mb, cov = m[4] - ma * mb;
            ssim += (2 * ma * mb + 1e-4) * (2 * cov + 9e-4) / ((ma * ma + mb * mb + 1e-4) * (va + vb + 9e-4));
            const double d = a[ty + kRadius][tx + kRadius] - b[ty + kRadius][tx + kRadius];
            l1 += fabs(d);
            sq += d * d;
        }
        __syncthreads();
    }
    ssim = warp_sum(ssim);
    l1 = warp_sum(l1);
    sq = warp_sum(sq);
    if ((t & 31) == 0) {
        red[0][t >> 5] = ssim;
        red[1][t >> 5] = l1;
        red[2][t >> 5] = sq;
    }
    __syncthreads();
    if (t < 3) {
        double s = 0.0;
        for (int k = 0; k < kEvalThreads / 32; ++k) s += red[t][k];
        partials[static_cast<size_t>(blockIdx.y * gridDim.x + blockIdx.x) * 3 + t] = s;
    }
}

// out[0..3] = PSNR (dB), mean SSIM, mean L1, MSE from the per-CTA partials.
__global__ void __launch_bounds__(kReduceThreads) eval_reduce_kernel(const double* __restrict__ partials, int blocks,
                                                                     double count, double* __restrict__ out) {
    __shared__ double red[3][kReduceThreads / 32];
    const int t = threadIdx.x;
    double s[3] = {0.0, 0.0, 0.0};
    for (int i = t; i < blocks; i += kReduceThreads)
#pragma unroll
        for (int j = 0; j < 3; ++j) s[j] += partials[static_cast<size_t>(i) * 3 + j];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        s[j] = warp_sum(s[j]);
        if ((t & 31) == 0) red[j][t >> 5] = s[j];
    }
    __syncthreads();
    if (t == 0) {
        double tot[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < kReduceThreads / 32; ++k)
            for (int j = 0; j < 3; ++j) tot[j] += red[j][k];
        const double mse = tot[2] / count;
        out[0] = mse > 0.0 ? -10.0 * log10(mse) : __longlong_as_double(0x7ff0000000000000LL);
        out[1] = tot[0] / count;
        out[2] = tot[1] / count;
        out[3] = mse;
    }
}

}  // namespace

size_t eval_metrics_workspace(int width, int height) {
    if (width <= 0 || height <= 0) return 0;
    const size_t blocks = static_cast<size_t>((width + kTileX - 1) / kTileX) * ((height + kTileY - 1) / kTileY);
    return blocks * 3 * sizeof(double);
}

int launch_eval_metrics(const float* image, const uint8_t* target, int width, int height, double* workspace,
                        double* out, cudaStream_t stream) {
    if (!image || !target || !workspace || !out || width <= 0 || height <= 0) return GSN_ERR_INVALID_ARGUMENT;
    Window win;
    double sum = 0.0;
    for (int k = 0; k < kTaps; ++k) {
        const double d = k - kRadius;
        win.w[k] = std::exp(-d * d / (2.0 * 1.5 * 1.5));
        sum += win.w[k];
    }
    for (int k = 0; k < kTaps; ++k) win.w[k] /= sum;
    const dim3 grid((width + kTileX - 1) / kTileX, (height + kTileY - 1) / kTileY);
    eval_metrics_kernel<<<grid, dim3(kTileX, kTileY), 0, stream>>>(image, target, width, height, win, workspace);
    eval_reduce_kernel<<<1, kReduceThreads, 0, stream>>>(workspace, static_cast<int>(grid.x * grid.y),
                                                         3.0 * static_cast<double>(width) * height, out);
    return launched(2);
}

}  // namespace gsn
