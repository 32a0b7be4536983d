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

#include <atomic>

namespace gsn {

namespace {

// Normalised 11-tap Gaussian, sigma 1.5 (the values of solver.cu:14-24).
__constant__ float c_window[11] = {1.028380120e-03f, 7.598758210e-03f, 3.600077330e-02f, 1.093606870e-01f,
                                   2.130055430e-01f, 2.660117150e-01f, 2.130055430e-01f, 1.093606870e-01f,
                                   3.600077330e-02f, 7.598758210e-03f, 1.028380120e-03f};

constexpr int kT = 32;                 // output tile edge
constexpr int kThreads = 256;
constexpr int kIn = kT + 20;           // raw input edge incl. the 10-pixel halo
constexpr int kCen = kT + 10;          // SSIM centres per edge incl. the 5-pixel halo
constexpr int kSeg1 = 7;               // outputs per thread in the moment passes (42 = 6 x 7)
constexpr int kSeg2 = 4;               // outputs per thread in the back-filter passes (32 = 8 x 4)
constexpr float kC1 = 0.0001f;
constexpr float kC2 = 0.0009f;
// shared arena (floats): raw image + target and five moment planes. The three
// partial planes reuse the raw planes once the horizontal pass has consumed them
// (each thread first copies its own output pixels' I and T to registers), and
// the back-filtered partials reuse the moment planes: 65 KB, three CTAs per SM.
constexpr int kRaw = kIn * kIn;
constexpr int kMom = kIn * kCen;
constexpr int kPart = kCen * kCen;
constexpr size_t kSmemBytes = sizeof(float) * (2 * kRaw + 5 * kMom);
static_assert(3 * kPart <= 2 * kRaw, "partials alias the raw planes");
static_assert((kT / kSeg2) * kT == kThreads, "one output column segment per thread");

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

// One block per 32x32 output tile and colour channel. Every filter output is
// produced by one thread from a register window of its row (or column), with
// the 11 taps accumulated in ascending order as in solver.cu:65-161.
__global__ void __launch_bounds__(kThreads, 3) loss_gradient_kernel(const float* __restrict__ image,
                                                                   const uint8_t* __restrict__ target_arg,
                                                                   const StepFrame* __restrict__ frame,
                                                                   float* __restrict__ grad, int width, int height,
                                                                   double* __restrict__ sums) {
    pdl_begin();
    extern __shared__ float smem[];
    const uint8_t* __restrict__ target = frame ? frame->target : target_arg;
    __shared__ double red[kThreads / 32];
    float* raw_i = smem;                 // [kIn][kIn]
    float* raw_t = raw_i + kRaw;         // [kIn][kIn]
    float* mom = raw_t + kRaw;           // [5][kIn][kCen]
    float* part = smem;                  // [3][kCen][kCen] (after the raw planes are consumed)
    float* back = mom;                   // [3][kCen][kT] (after the moments are consumed)
    const int t = threadIdx.x;
    const int ch = blockIdx.z;
    const int ox = blockIdx.x * kT, oy = blockIdx.y * kT;

    // raw inputs with a zero-padded halo: all of a thread's loads are issued
    // before the first shared-memory store, so they are in flight together
    {
        constexpr int kRawPer = (kRaw + kThreads - 1) / kThreads;
        float ri[kRawPer], rt[kRawPer];
#pragma unroll
        for (int u = 0; u < kRawPer; ++u) {
            const int j = t + u * kThreads;
            const int hx = ox + j % kIn - 10, hy = oy + j / kIn - 10;
            const bool ok = j < kRaw && hx >= 0 && hy >= 0 && hx < width && hy < height;
            const int64_t k = (static_cast<int64_t>(hy) * width + hx) * 3 + ch;
            ri[u] = ok ? image[k] : 0.0f;
            rt[u] = ok ? target[k] * (1.0f / 255.0f) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kRawPer; ++u) {
            const int j = t + u * kThreads;
            if (j < kRaw) {
                raw_i[j] = ri[u];
                raw_t[j] = rt[u];
            }
        }
    }
    __syncthreads();

    // horizontal pass over the five moments: kIn rows x kCen centres
    for (int item = t; item < kIn * (kCen / kSeg1); item += kThreads) {
        const int r = item / (kCen / kSeg1);
        const int c0 = (item % (kCen / kSeg1)) * kSeg1;
        float a[kSeg1 + 10], b[kSeg1 + 10];
#pragma unroll
        for (int k = 0; k < kSeg1 + 10; ++k) {
            a[k] = raw_i[r * kIn + c0 + k];
            b[k] = raw_t[r * kIn + c0 + k];
        }
#pragma unroll
        for (int o = 0; o < kSeg1; ++o) {
            float h0 = 0.f, h1 = 0.f, h2 = 0.f, h3 = 0.f, h4 = 0.f;
#pragma unroll
            for (int dx = 0; dx < 11; ++dx) {
                float w = c_window[dx];
                float av = a[o + dx], bv = b[o + dx];
                h0 += w * av;
                h1 += w * bv;
                h2 += w * av * av;
                h3 += w * bv * bv;
                h4 += w * av * bv;
            }
            const int idx = r * kCen + c0 + o;
            mom[0 * kMom + idx] = h0;
            mom[1 * kMom + idx] = h1;
            mom[2 * kMom + idx] = h2;
            mom[3 * kMom + idx] = h3;
            mom[4 * kMom + idx] = h4;
        }
    }
    __syncthreads();
    // this thread's output pixels (column x_out, rows y_out .. y_out + 3) of the
    // raw planes, kept in registers before the partials overwrite them
    const int x_out = t % kT, y_out = (t / kT) * kSeg2;
    float keep_i[kSeg2], keep_t[kSeg2];
#pragma unroll
    for (int o = 0; o < kSeg2; ++o) {
        keep_i[o] = raw_i[(y_out + o + 10) * kIn + x_out + 10];
        keep_t[o] = raw_t[(y_out + o + 10) * kIn + x_out + 10];
    }
    __syncthreads();

    // vertical pass -> moments at the centres, then the SSIM partials
    double ssim_sum = 0.0;
    for (int item = t; item < (kCen / kSeg1) * kCen; item += kThreads) {
        const int cx = item % kCen;
        const int r0 = (item / kCen) * kSeg1;
        float M[5][kSeg1];
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            float col[kSeg1 + 10];
#pragma unroll
            for (int k = 0; k < kSeg1 + 10; ++k) col[k] = mom[m * kMom + (r0 + k) * kCen + cx];
#pragma unroll
            for (int o = 0; o < kSeg1; ++o) {
                float acc = 0.0f;
#pragma unroll
                for (int dy = 0; dy < 11; ++dy) acc += c_window[dy] * col[o + dy];
                M[m][o] = acc;
            }
        }
        const int hx = ox + cx - 5;
#pragma unroll
        for (int o = 0; o < kSeg1; ++o) {
            const int cy = r0 + o;
            const int hy = oy + cy - 5;
            float pa = 0.0f, pb = 0.0f, pc = 0.0f;
            if (hx >= 0 && hy >= 0 && hx < width && hy < height) {
                float m = M[0][o], n = M[1][o];
                float inv_d = 1.0f / (m * m + n * n + kC1);
                float inv_e = 1.0f / (M[2][o] - m * m + M[3][o] - n * n + kC2);
                float lum = (2 * m * n + kC1) * inv_d;
                float cs = (2 * (M[4][o] - m * n) + kC2) * inv_e;
                float dmu = 2 * (n - m * lum) * inv_d * cs;
                pb = 2 * lum * inv_e;
                pc = -lum * cs * inv_e;
                pa = dmu - n * pb - 2 * m * pc;
                if (sums && cx >= 5 && cx < 5 + kT && cy >= 5 && cy < 5 + kT)
                    ssim_sum += static_cast<double>(lum) * static_cast<double>(cs);
            }
            const int idx = cy * kCen + cx;
            part[0 * kPart + idx] = pa;
            part[1 * kPart + idx] = pb;
            part[2 * kPart + idx] = pc;
        }
    }
    __syncthreads();

    // horizontal back-filter of the partials: kCen rows x kT columns
    for (int item = t; item < kCen * (kT / kSeg2); item += kThreads) {
        const int r = item / (kT / kSeg2);
        const int c0 = (item % (kT / kSeg2)) * kSeg2;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
            float v[kSeg2 + 10];
#pragma unroll
            for (int k = 0; k < kSeg2 + 10; ++k) v[k] = part[p * kPart + r * kCen + c0 + k];
#pragma unroll
            for (int o = 0; o < kSeg2; ++o) {
                float acc = 0.0f;
#pragma unroll
                for (int dx = 0; dx < 11; ++dx) acc += c_window[dx] * v[o + dx];
                back[p * kCen * kT + r * kT + c0 + o] = acc;
            }
        }
    }
    __syncthreads();

    // vertical back-filter at the output pixels and the combined gradient
    double l1_sum = 0.0, sq_sum = 0.0;
    const float norm = 1.0f / (3.0f * static_cast<float>(width) * height);
    {
        const int x = x_out;
        const int y0 = y_out;
        float f[3][kSeg2];
#pragma unroll
        for (int p = 0; p < 3; ++p) {
            float v[kSeg2 + 10];
#pragma unroll
            for (int k = 0; k < kSeg2 + 10; ++k) v[k] = back[p * kCen * kT + (y0 + k) * kT + x];
#pragma unroll
            for (int o = 0; o < kSeg2; ++o) {
                float acc = 0.0f;
#pragma unroll
                for (int dy = 0; dy < 11; ++dy) acc += c_window[dy] * v[o + dy];
                f[p][o] = acc;
            }
        }
#pragma unroll
        for (int o = 0; o < kSeg2; ++o) {
            const int px = ox + x, py = oy + y0 + o;
            if (px < width && py < height) {
                const float I = keep_i[o];
                const float R = keep_t[o];
                float r = I - R;
                float l1 = static_cast<float>(r > 0) - static_cast<float>(r < 0);
                float dssim = -(f[0][o] + R * f[1][o] + 2 * I * f[2][o]);
                grad[(static_cast<int64_t>(py) * width + px) * 3 + ch] = (0.8f * l1 + 0.2f * dssim) * norm;
                if (sums) {
                    double d = static_cast<double>(I) - static_cast<double>(R);
                    l1_sum += fabs(d);
                    sq_sum += d * d;
                }
            }
        }
    }
    if (sums) {
        double l1s = block_sum(l1_sum, red);
        double sq = block_sum(sq_sum, red);
        double ss = block_sum(ssim_sum, red);
        if (t == 0) {
            atomicAdd(sums + 0, l1s);
            atomicAdd(sums + 1, ss);
            atomicAdd(sums + 2, sq);
        }
    }
}

__device__ __forceinline__ float2 pk(float a) { return make_float2(a, a); }

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Fast form: the same tiles and passes with two of the filtered quantities
// packed into one FP32x2 FMA chain wherever they share the window (sm_100
// packed arithmetic, each half rounded as its scalar FMA): (I, T) and
// (I^2, T^2) in the moment passes, the partials (dSSIM/dmu, dSSIM/dE[xy]) in
// the back-filter passes; E[I T] and dSSIM/dE[x^2] stay scalar. Each product
// is formed once per input, every filter output is one 11-FMA chain from zero,
// and the per-centre SSIM partials use the hardware reciprocal approximation.
// The shared arena holds the same planes interleaved: (I, T) raw pairs, (mu_I,
// mu_T) and (E[I^2], E[T^2]) row-filtered pairs and the scalar E[I T] plane;
// the partials alias the raw pairs, the back-filtered partials the moments.
__global__ void __launch_bounds__(kThreads, 3) loss_gradient_fast_kernel(const float* __restrict__ image,
                                                                        const uint8_t* __restrict__ target_arg,
                                                                        const StepFrame* __restrict__ frame,
                                                                        float* __restrict__ grad, int width,
                                                                        int height, double* __restrict__ sums) {
    pdl_begin();
    extern __shared__ float smem[];
    const uint8_t* __restrict__ target = frame ? frame->target : target_arg;
    __shared__ double red[kThreads / 32];
    float2* raw = reinterpret_cast<float2*>(smem);               // [kIn][kIn] (I, T)
    float2* mom01 = reinterpret_cast<float2*>(smem + 2 * kRaw);  // [kIn][kCen] (I, T) row-filtered
    float2* mom23 = mom01 + kMom;                                // [kIn][kCen] (I^2, T^2)
    float* mom4 = reinterpret_cast<float*>(mom23 + kMom);        // [kIn][kCen] I T
    float2* part01 = raw;                                        // [kCen][kCen] (pa, pb)
    float* part2 = reinterpret_cast<float*>(part01 + kPart);     // [kCen][kCen] pc
    float2* back01 = mom01;                                      // [kCen][kT]
    float* back2 = reinterpret_cast<float*>(back01 + kCen * kT); // [kCen][kT]
    const int t = threadIdx.x;
    const int ch = blockIdx.z;
    const int ox = blockIdx.x * kT, oy = blockIdx.y * kT;

    {
        constexpr int kRawPer = (kRaw + kThreads - 1) / kThreads;
        float ri[kRawPer], rt[kRawPer];
#pragma unroll
        for (int u = 0; u < kRawPer; ++u) {
            const int j = t + u * kThreads;
            const int hx = ox + j % kIn - 10, hy = oy + j / kIn - 10;
            const bool ok = j < kRaw && hx >= 0 && hy >= 0 && hx < width && hy < height;
            const int64_t k = (static_cast<int64_t>(hy) * width + hx) * 3 + ch;
            ri[u] = ok ? image[k] : 0.0f;
            rt[u] = ok ? target[k] * (1.0f / 255.0f) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kRawPer; ++u) {
            const int j = t + u * kThreads;
            if (j < kRaw) raw[j] = make_float2(ri[u], rt[u]);
        }
    }
    __syncthreads();

    // horizontal pass: kIn rows x kCen centres
    for (int item = t; item < kIn * (kCen / kSeg1); item += kThreads) {
        const int r = item / (kCen / kSeg1);
        const int c0 = (item % (kCen / kSeg1)) * kSeg1;
        const int row = r * kCen + c0;
        float2 v[kSeg1 + 10];
#pragma unroll
        for (int k = 0; k < kSeg1 + 10; ++k) v[k] = raw[r * kIn + c0 + k];
#pragma unroll
        for (int o = 0; o < kSeg1; ++o) {
            float2 acc = pk(0.0f);
#pragma unroll
            for (int dx = 0; dx < 11; ++dx) acc = __ffma2_rn(pk(c_window[dx]), v[o + dx], acc);
            mom01[row + o] = acc;
        }
        float2 sq[kSeg1 + 10];
#pragma unroll
        for (int k = 0; k < kSeg1 + 10; ++k) sq[k] = __fmul2_rn(v[k], v[k]);
#pragma unroll
        for (int o = 0; o < kSeg1; ++o) {
            float2 acc = pk(0.0f);
#pragma unroll
            for (int dx = 0; dx < 11; ++dx) acc = __ffma2_rn(pk(c_window[dx]), sq[o + dx], acc);
            mom23[row + o] = acc;
        }
#pragma unroll
        for (int o = 0; o < kSeg1; ++o) {
            float acc = 0.0f;
#pragma unroll
            for (int dx = 0; dx < 11; ++dx) acc = fmaf(c_window[dx], v[o + dx].x * v[o + dx].y, acc);
            mom4[row + o] = acc;
        }
    }
    __syncthreads();
    const int x_out = t % kT, y_out = (t / kT) * kSeg2;
    float2 keep[kSeg2];
#pragma unroll
    for (int o = 0; o < kSeg2; ++o) keep[o] = raw[(y_out + o + 10) * kIn + x_out + 10];
    __syncthreads();

    // vertical pass -> moments at the centres, then the SSIM partials
    double ssim_sum = 0.0;
    for (int item = t; item < (kCen / kSeg1) * kCen; item += kThreads) {
        const int cx = item % kCen;
        const int r0 = (item / kCen) * kSeg1;
        float2 M01[kSeg1], M23[kSeg1];
        float M4[kSeg1];
        {
            float2 col[kSeg1 + 10];
#pragma unroll
            for (int k = 0; k < kSeg1 + 10; ++k) col[k] = mom01[(r0 + k) * kCen + cx];
#pragma unroll
            for (int o = 0; o < kSeg1; ++o) {
                float2 acc = pk(0.0f);
#pragma unroll
                for (int dy = 0; dy < 11; ++dy) acc = __ffma2_rn(pk(c_window[dy]), col[o + dy], acc);
                M01[o] = acc;
            }
        }
        {
            float2 col[kSeg1 + 10];
#pragma unroll
            for (int k = 0; k < kSeg1 + 10; ++k) col[k] = mom23[(r0 + k) * kCen + cx];
#pragma unroll
            for (int o = 0; o < kSeg1; ++o) {
                float2 acc = pk(0.0f);
#pragma unroll
                for (int dy = 0; dy < 11; ++dy) acc = __ffma2_rn(pk(c_window[dy]), col[o + dy], acc);
                M23[o] = acc;
            }
        }
        {
            float col[kSeg1 + 10];
#pragma unroll
            for (int k = 0; k < kSeg1 + 10; ++k) col[k] = mom4[(r0 + k) * kCen + cx];
#pragma unroll
            for (int o = 0; o < kSeg1; ++o) {
                float acc = 0.0f;
#pragma unroll
                for (int dy = 0; dy < 11; ++dy) acc = fmaf(c_window[dy], col[o + dy], acc);
                M4[o] = acc;
            }
        }
        const int hx = ox + cx - 5;
#pragma unroll
        for (int o = 0; o < kSeg1; ++o) {
            const int cy = r0 + o;
            const int hy = oy + cy - 5;
            float pa = 0.0f, pb = 0.0f, pc = 0.0f;
            if (hx >= 0 && hy >= 0 && hx < width && hy < height) {
                const float m = M01[o].x, n = M01[o].y;
                const float inv_d = rcp_approx(m * m + n * n + kC1);
                const float inv_e = rcp_approx(M23[o].x - m * m + M23[o].y - n * n + kC2);
                const float lum = (2 * m * n + kC1) * inv_d;
                const float cs = (2 * (M4[o] - m * n) + kC2) * inv_e;
                const float dmu = 2 * (n - m * lum) * inv_d * cs;
                pb = 2 * lum * inv_e;
                pc = -lum * cs * inv_e;
                pa = dmu - n * pb - 2 * m * pc;
                if (sums && cx >= 5 && cx < 5 + kT && cy >= 5 && cy < 5 + kT)
                    ssim_sum += static_cast<double>(lum) * static_cast<double>(cs);
            }
            const int idx = cy * kCen + cx;
            part01[idx] = make_float2(pa, pb);
            part2[idx] = pc;
        }
    }
    __syncthreads();

    // horizontal back-filter of the partials: kCen rows x kT columns
    for (int item = t; item < kCen * (kT / kSeg2); item += kThreads) {
        const int r = item / (kT / kSeg2);
        const int c0 = (item % (kT / kSeg2)) * kSeg2;
        {
            float2 v[kSeg2 + 10];
#pragma unroll
            for (int k = 0; k < kSeg2 + 10; ++k) v[k] = part01[r * kCen + c0 + k];
#pragma unroll
            for (int o = 0; o < kSeg2; ++o) {
                float2 acc = pk(0.0f);
#pragma unroll
                for (int dx = 0; dx < 11; ++dx) acc = __ffma2_rn(pk(c_window[dx]), v[o + dx], acc);
                back01[r * kT + c0 + o] = acc;
            }
        }
        {
            float v[kSeg2 + 10];
#pragma unroll
            for (int k = 0; k < kSeg2 + 10; ++k) v[k] = part2[r * kCen + c0 + k];
#pragma unroll
            for (int o = 0; o < kSeg2; ++o) {
                float acc = 0.0f;
#pragma unroll
                for (int dx = 0; dx < 11; ++dx) acc = fmaf(c_window[dx], v[o + dx], acc);
                back2[r * kT + c0 + o] = acc;
            }
        }
    }
    __syncthreads();

    // vertical back-filter at the output pixels and the combined gradient
    double l1_sum = 0.0, sq_sum = 0.0;
    const float norm = 1.0f / (3.0f * static_cast<float>(width) * height);
    float2 f01[kSeg2];
    float f2[kSeg2];
    {
        float2 v[kSeg2 + 10];
#pragma unroll
        for (int k = 0; k < kSeg2 + 10; ++k) v[k] = back01[(y_out + k) * kT + x_out];
#pragma unroll
        for (int o = 0; o < kSeg2; ++o) {
            float2 acc = pk(0.0f);
#pragma unroll
            for (int dy = 0; dy < 11; ++dy) acc = __ffma2_rn(pk(c_window[dy]), v[o + dy], acc);
            f01[o] = acc;
        }
    }
    {
        float v[kSeg2 + 10];
#pragma unroll
        for (int k = 0; k < kSeg2 + 10; ++k) v[k] = back2[(y_out + k) * kT + x_out];
#pragma unroll
        for (int o = 0; o < kSeg2; ++o) {
            float acc = 0.0f;
#pragma unroll
            for (int dy = 0; dy < 11; ++dy) acc = fmaf(c_window[dy], v[o + dy], acc);
            f2[o] = acc;
        }
    }
#pragma unroll
    for (int o = 0; o < kSeg2; ++o) {
        const int px = ox + x_out, py = oy + y_out + o;
        if (px < width && py < height) {
            const float I = keep[o].x;
            const float R = keep[o].y;
            const float r = I - R;
            const float l1 = static_cast<float>(r > 0) - static_cast<float>(r < 0);
            const float dssim = -(f01[o].x + R * f01[o].y + 2 * I * f2[o]);
            grad[(static_cast<int64_t>(py) * width + px) * 3 + ch] = (0.8f * l1 + 0.2f * dssim) * norm;
            if (sums) {
                const double d = static_cast<double>(I) - static_cast<double>(R);
                l1_sum += fabs(d);
                sq_sum += d * d;
            }
        }
    }
    if (sums) {
        double l1s = block_sum(l1_sum, red);
        double sq = block_sum(sq_sum, red);
        double ss = block_sum(ssim_sum, red);
        if (t == 0) {
            atomicAdd(sums + 0, l1s);
            atomicAdd(sums + 1, ss);
            atomicAdd(sums + 2, sq);
        }
    }
}

__global__ void finalize_loss_kernel(const double* sums, int width, int height, double* out) {
    pdl_begin();
    double count = 3.0 * static_cast<double>(width) * height;
    double l1 = sums[0] / count, ssim = sums[1] / count, mse = sums[2] / count;
    out[0] = 0.8 * l1 + 0.2 * (1.0 - ssim);
    out[1] = l1;
    out[2] = ssim;
    out[3] = mse > 0.0 ? -10.0 * log10(mse) : INFINITY;
}

}  // namespace

int launch_loss_gradient(const float* image, const uint8_t* target, const StepFrame* frame, float* grad, int width,
                         int height, double* sums, cudaStream_t stream, bool fast) {
    if (width <= 0 || height <= 0) return GSN_ERR_INVALID_ARGUMENT;
    if (sums && cudaMemsetAsync(sums, 0, 3 * sizeof(double), stream) != cudaSuccess) return GSN_ERR_CUDA;
    // the dynamic shared-memory opt-in is a per-device, per-kernel attribute
    // set once per device and form; concurrent host threads may both set it
    static std::atomic<bool> configured[64][2] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return GSN_ERR_CUDA;
    if (device < 0 || device >= 64) return GSN_ERR_CUDA;
    if (!configured[device][fast ? 1 : 0].load()) {
        const cudaError_t e =
            fast ? cudaFuncSetAttribute(loss_gradient_fast_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(kSmemBytes))
                 : cudaFuncSetAttribute(loss_gradient_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(kSmemBytes));
        if (e != cudaSuccess) return GSN_ERR_CUDA;
        configured[device][fast ? 1 : 0].store(true);
    }
    dim3 grid(ceil_div(width, kT), ceil_div(height, kT), 3);
    if (fast)
        launch_step(loss_gradient_fast_kernel, grid, kThreads, kSmemBytes, stream, image, target, frame, grad, width,
                    height, sums);
    else
        launch_step(loss_gradient_kernel, grid, kThreads, kSmemBytes, stream, image, target, frame, grad, width, height,
                    sums);
    return launched(1);
}

int launch_finalize_loss(const double* sums, int width, int height, double* out, cudaStream_t stream) {
    launch_step(finalize_loss_kernel, 1, 1, 0, stream, sums, width, height, out);
    return launched(1);
}

}  // namespace gsn
