// Minimal OpenCV-compatible image filtering for the reference's CPU reference
// loss (test/cpu_reference.h ComputeLoss): getGaussianKernel and sepFilter2D
// with a constant zero border. TEST INFRASTRUCTURE ONLY (oracle/).
#pragma once

#include <algorithm>
#include <cmath>

#include "core.hpp"

#define CV_PI 3.1415926535897932384626433832795

namespace cv {

enum BorderTypes { BORDER_CONSTANT = 0 };

// ksize x 1 kernel of G_i = a * exp(-(i - (ksize - 1) / 2)^2 / (2 sigma^2)),
// a chosen so that the taps sum to 1 (the documented definition; for
// sigma <= 0 the documented default sigma = 0.3 ((ksize - 1) / 2 - 1) + 0.8).
inline Mat getGaussianKernel(int ksize, double sigma, int ktype = CV_64F) {
    const double s = sigma > 0 ? sigma : ((ksize - 1) * 0.5 - 1) * 0.3 + 0.8;
    const double scale = -0.5 / (s * s);
    std::vector<double> taps(ksize);
    double sum = 0;
    for (int i = 0; i < ksize; ++i) {
        const double x = i - (ksize - 1) * 0.5;
        taps[i] = std::exp(scale * x * x);
        sum += taps[i];
    }
    Mat k(ksize, 1, CV_MAKETYPE(ktype, 1));
    for (int i = 0; i < ksize; ++i) k.set(i, 0, 0, taps[i] / sum);
    return k;
}

// dst(y, x) = sum_j ky[j] * sum_i kx[i] * src(y + j - ay, x + i - ax) + delta per
// channel (correlation, anchor at the kernel centre when negative), samples
// outside the image read as 0 (BORDER_CONSTANT); the row pass runs first.
inline void sepFilter2D(const Mat& src, Mat& dst, int ddepth, const Mat& kernelX, const Mat& kernelY,
                        Point anchor = Point(-1, -1), double delta = 0, int borderType = BORDER_CONSTANT) {
    if (borderType != BORDER_CONSTANT) throw std::runtime_error("cv shim: only BORDER_CONSTANT");
    const int kx = static_cast<int>(kernelX.total()), ky = static_cast<int>(kernelY.total());
    const int ax = anchor.x < 0 ? kx / 2 : anchor.x, ay = anchor.y < 0 ? ky / 2 : anchor.y;
    const int cn = src.channels(), W = src.cols, H = src.rows;
    std::vector<double> wx(kx), wy(ky);
    for (int i = 0; i < kx; ++i) wx[i] = kernelX.get(kernelX.rows == 1 ? 0 : i, kernelX.rows == 1 ? i : 0, 0);
    for (int j = 0; j < ky; ++j) wy[j] = kernelY.get(kernelY.rows == 1 ? 0 : j, kernelY.rows == 1 ? j : 0, 0);
    // interleaved channels as doubles, then the row pass and the column pass
    const size_t row = static_cast<size_t>(W) * cn;
    std::vector<double> in(static_cast<size_t>(H) * row), mid(in.size());
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int k = 0; k < cn; ++k) in[y * row + static_cast<size_t>(x) * cn + k] = src.get(y, x, k);
    for (int y = 0; y < H; ++y) {
        const double* s = in.data() + y * row;
        double* m = mid.data() + y * row;
        for (int x = 0; x < W; ++x) {
            const int i0 = ax - x > 0 ? ax - x : 0, i1 = W - x + ax < kx ? W - x + ax : kx;
            for (int k = 0; k < cn; ++k) {
                double acc = 0;
                for (int i = i0; i < i1; ++i) acc += wx[i] * s[static_cast<size_t>(x + i - ax) * cn + k];
                m[static_cast<size_t>(x) * cn + k] = acc;
            }
        }
    }
    Mat out(H, W, CV_MAKETYPE(ddepth < 0 ? src.depth() : ddepth, cn));
    std::vector<double> acc(row);
    for (int y = 0; y < H; ++y) {
        std::fill(acc.begin(), acc.end(), 0.0);
        for (int j = 0; j < ky; ++j) {
            const int yy = y + j - ay;
            if (yy < 0 || yy >= H) continue;
            const double* m = mid.data() + yy * row;
            for (size_t e = 0; e < row; ++e) acc[e] += wy[j] * m[e];
        }
        for (int x = 0; x < W; ++x)
            for (int k = 0; k < cn; ++k) out.set(y, x, k, acc[static_cast<size_t>(x) * cn + k] + delta);
    }
    dst = out;
}

}  // namespace cv
