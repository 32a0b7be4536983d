// gsn_render: renders a trained PLY model from the train or test views of a
// COLMAP scene and writes <output>/<split>/gs-native/{renders,gt,comparison}/
// NNNNN.png and psnr.csv (per-view 8-bit PSNR and the mean), as the
// reference's demo/render.cpp:21-160 does, without OpenCV. metrics.csv adds
// the FP64 held-out-view metrics computed on the GPU (render clamped to
// [0, 1]: PSNR of the RGB MSE, 11x11 Gaussian SSIM, L1) per view and their mean.
//
//   gsn_render --scene DIR --model PLY --output DIR [--downscale 1]
//              [--sh_degree 3] [--split test]
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <vector>

#include "args.h"
#include "core/render/renderer.h"
#include "io/colmap.h"
#include "io/ply.h"
#include "kernels.h"

int main(int argc, char** argv) {
    gs_native_demo::Args args(argc, argv,
                              {{"scene", ""},
                               {"model", ""},
                               {"output", ""},
                               {"downscale", "1"},
                               {"sh_degree", "3"},
                               {"split", "test"}});
    if (args.help()) {
        args.usage("gs-native B200 rendering");
        return 0;
    }
    const std::string split = args.error().empty() ? args.str("split") : "";
    if (!args.error().empty() || (split != "test" && split != "train")) {
        std::cerr << args.error() << "\nSpecify --scene, --model, --output and --split=test or train.\n";
        return 1;
    }
    const int downscale = std::max(1, args.integer("downscale"));
    const int sh_degree = std::clamp(args.integer("sh_degree"), 0, 3);

    gs_native::ColmapScene scene;
    std::vector<gs_native::Gaussian> gaussians;
    if (!gs_native::ReadColmapScene(args.str("scene"), downscale, scene) ||
        !gs_native::ReadGaussiansPly(args.str("model"), gaussians)) {
        std::cerr << "Reading the scene or the model failed.\n";
        return 1;
    }
    const auto& cameras = split == "test" ? scene.test_cameras : scene.train_cameras;
    const auto& targets = split == "test" ? scene.test_images : scene.train_images;
    const auto& names = split == "test" ? scene.test_names : scene.train_names;
    if (cameras.empty() || gaussians.empty() ||
        gaussians.size() > static_cast<size_t>(std::numeric_limits<int>::max())) {
        std::cerr << "No cameras or no valid Gaussians.\n";
        return 1;
    }
    const int count = static_cast<int>(gaussians.size());
    const std::vector<float> params = gs_native::PackGaussians(gaussians);
    size_t pixels = 0;
    size_t workspace = 0;  // FP64 metric partials
    for (const auto& t : targets) {
        pixels = std::max(pixels, static_cast<size_t>(t.width) * t.height);
        workspace = std::max(workspace, gsn::eval_metrics_workspace(t.width, t.height));
    }

    int result = 0;
    float* device_params = nullptr;
    float* device_image = nullptr;
    uint8_t* device_target = nullptr;
    double* device_metrics = nullptr;
    try {
        if (cudaMalloc(&device_params, params.size() * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&device_image, pixels * 3 * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&device_target, pixels * 3) != cudaSuccess ||
            cudaMalloc(&device_metrics, 4 * sizeof(double) + workspace) != cudaSuccess ||
            cudaMemcpy(device_params, params.data(), params.size() * sizeof(float), cudaMemcpyHostToDevice) !=
                cudaSuccess)
            throw std::runtime_error("Allocating or uploading rendering buffers failed.");
        const std::filesystem::path destination = std::filesystem::path(args.str("output")) / split / "gs-native";
        if (std::filesystem::exists(destination) && !std::filesystem::is_empty(destination))
            throw std::runtime_error("Rendering directory is not empty: " + destination.string());
        for (const char* d : {"renders", "gt", "comparison"}) std::filesystem::create_directories(destination / d);
        std::ofstream report(destination / "psnr.csv");
        if (!report) throw std::runtime_error("Opening PSNR report failed.");
        report << "image,psnr_db\n" << std::setprecision(10);
        std::ofstream metrics(destination / "metrics.csv");
        if (!metrics) throw std::runtime_error("Opening metrics report failed.");
        metrics << "image,psnr_db,ssim,l1\n" << std::setprecision(12);
        double metric_sums[3] = {0.0, 0.0, 0.0};

        gs_native::GaussianBuffers buffers;
        buffers.gaussians_ = device_params;
        buffers.gaussian_count_ = count;
        gs_native::Renderer renderer;
        const float background[3] = {0.0f, 0.0f, 0.0f};
        std::vector<float> image;
        double sum = 0;
        for (size_t i = 0; i < cameras.size(); ++i) {
            const gs_native::CameraParams& camera = cameras[i];
            const size_t n = static_cast<size_t>(camera.width_) * camera.height_ * 3;
            image.resize(n);
            if (!renderer.Render(buffers, camera, background, device_image, sh_degree) ||
                cudaMemcpy(image.data(), device_image, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
                throw std::runtime_error("Rendering failed at " + names[i]);
            double m[4];
            if (cudaMemcpy(device_target, targets[i].rgb.data(), n, cudaMemcpyHostToDevice) != cudaSuccess ||
                gsn::launch_eval_metrics(device_image, device_target, camera.width_, camera.height_,
                                         device_metrics + 4, device_metrics, nullptr) != GSN_OK ||
                cudaMemcpy(m, device_metrics, sizeof(m), cudaMemcpyDeviceToHost) != cudaSuccess)
                throw std::runtime_error("Evaluating failed at " + names[i]);
            for (int q = 0; q < 3; ++q) metric_sums[q] += m[q];
            gs_native::ImageU8 render;
            render.width = camera.width_;
            render.height = camera.height_;
            render.rgb.resize(n);
            double squared = 0;
            for (size_t k = 0; k < n; ++k) {
                if (!std::isfinite(image[k])) throw std::runtime_error("Non-finite pixel at " + names[i]);
                const float v = std::min(std::max(image[k], 0.0f), 1.0f) * 255.0f;
                render.rgb[k] = static_cast<uint8_t>(std::lrint(v));
                const double d = static_cast<double>(render.rgb[k]) - targets[i].rgb[k];
                squared += d * d;
            }
            const double mse = squared / (static_cast<double>(n) * 255.0 * 255.0);
            const double psnr = mse == 0 ? std::numeric_limits<double>::infinity() : -10.0 * std::log10(mse);
            sum += psnr;
            char name[32];
            std::snprintf(name, sizeof(name), "%05d.png", static_cast<int>(i));
            report << name << ',' << psnr << '\n';
            metrics << name << ',' << m[0] << ',' << m[1] << ',' << m[2] << '\n';
            if (!gs_native::WritePng((destination / "renders" / name).string(), render) ||
                !gs_native::WritePng((destination / "gt" / name).string(), targets[i]) ||
                !gs_native::WritePng((destination / "comparison" / name).string(),
                                     gs_native::ConcatHorizontal(render, targets[i])))
                throw std::runtime_error("Saving rendered image failed.");
            std::cout << "View " << i << " (" << names[i] << "): PSNR " << std::fixed << std::setprecision(6) << psnr
                      << " dB" << std::endl;
        }
        metrics << "mean," << metric_sums[0] / cameras.size() << ',' << metric_sums[1] / cameras.size() << ','
                << metric_sums[2] / cameras.size() << '\n';
        metrics.close();
        if (!metrics) throw std::runtime_error("Writing metrics report failed.");
        report << "mean," << sum / cameras.size() << '\n';
        report.close();
        if (!report) throw std::runtime_error("Writing PSNR report failed.");
        std::cout << "Mean PSNR: " << sum / cameras.size() << " dB (8-bit), FP64 PSNR "
                  << metric_sums[0] / cameras.size() << " dB, SSIM " << metric_sums[1] / cameras.size()
                  << "\nOutput: " << destination.string() << std::endl;
    } catch (const std::exception& error) {
        std::cerr << error.what() << '\n';
        result = 1;
    }
    cudaFree(device_metrics);
    cudaFree(device_target);
    cudaFree(device_image);
    cudaFree(device_params);
    return result;
}
