// Test-infrastructure harness: the reference's CPU reference renderer and loss
// (test/cpu_reference.h RenderReference and ComputeLoss, compiled unmodified
// from the reference tree against the OpenCV shim in oracle/cv_shim) behind
// extern "C" entry points. Used by the CPU tests as a second oracle and by the
// benchmark's CPU baseline; not part of the product.
#include "cpu_reference.h"

#include <cstring>

using gs_native::CameraParams;
using gs_native::Gaussian;

namespace {

// The 58 x count SoA parameter block (buffers.h:10-15) as the reference's
// host Gaussians (the inverse of PackGaussians, test_support.h:84-100).
std::vector<Gaussian> Unpack(const float* params, int count) {
    std::vector<Gaussian> out(static_cast<size_t>(count));
    const size_t n = static_cast<size_t>(count);
    for (size_t i = 0; i < n; ++i) {
        Gaussian& g = out[i];
        for (int a = 0; a < 3; ++a) {
            g.position_[a] = params[a * n + i];
            g.log_scale_[a] = params[(gs_native::kLogScaleIndex + a) * n + i];
            g.rotation_[a] = params[(gs_native::kRotationIndex + a) * n + i];
            for (int k = 0; k < 16; ++k) g.sh_(k, a) = params[(gs_native::kShIndex + a * 16 + k) * n + i];
        }
        g.opacity_logit_ = params[gs_native::kOpacityIndex * n + i];
    }
    return out;
}

}  // namespace

extern "C" {

// RenderReference (cpu_reference.h:22-116): FP64 HWC RGB image of
// camera->height_ x camera->width_ pixels into `image`.
int ref_cpu_render(const float* params, int count, const CameraParams* camera, const float* background, int degree,
                   double* image) {
    try {
        std::array<float, 3> bg = {background[0], background[1], background[2]};
        cv::Mat out = gs_native::test::RenderReference(Unpack(params, count), *camera, bg, degree);
        for (int y = 0; y < out.rows; ++y)
            std::memcpy(image + static_cast<size_t>(y) * out.cols * 3, out.data + y * out.step,
                        static_cast<size_t>(out.cols) * 3 * sizeof(double));
        return 0;
    } catch (...) {
        return -1;
    }
}

// ComputeLoss (cpu_reference.h:118-152) of an FP64 HWC RGB image against a u8
// HWC RGB target.
int ref_cpu_loss(const double* image, const uint8_t* target, int width, int height, double* loss) {
    try {
        cv::Mat img(height, width, CV_64FC3, const_cast<double*>(image));
        cv::Mat tgt(height, width, CV_8UC3, const_cast<uint8_t*>(target));
        *loss = gs_native::test::ComputeLoss(img, tgt);
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
