// gsn_train: trains a model on a COLMAP scene and writes
// <output>/point_cloud/iteration_<N>/point_cloud.ply plus a viewer cfg_args,
// as the reference's demo/train.cpp:15-110 does, without OpenCV (images are
// pre-decoded PPM files, see io/colmap.h).
//
//   gsn_train --scene DIR --output DIR [--downscale 1] [--iterations 30000]
//             [--precision] [--graph] [--max_gaussians 0]
//             [--culled] [--sparse] [--fast] [--fp32_ssim]
//             [--checkpoint PATH] [--resume PATH]
//
// --culled: exact tile culling; --sparse: visibility-masked Adam on the
// Morton-ordered model; --fast: the fast blend arithmetic; --fp32_ssim: with
// --precision, the fp32 SSIM gradient instead of the tcgen05 one. All four with
// --precision and --graph give the fastest form.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>

#include "args.h"
#include "core/gaussian_splatting.h"
#include "io/colmap.h"

namespace {

double Seconds(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

int main(int argc, char** argv) {
    gs_native_demo::Args args(argc, argv,
                              {{"scene", ""},
                               {"output", ""},
                               {"downscale", "1"},
                               {"iterations", "30000"},
                               {"precision", "false"},
                               {"graph", "false"},
                               {"max_gaussians", "0"},
                               {"culled", "false"},
                               {"sparse", "false"},
                               {"fast", "false"},
                               {"fp32_ssim", "false"},
                               {"checkpoint", "none"},
                               {"resume", "none"}});
    if (args.help()) {
        args.usage("gs-native B200 training");
        return 0;
    }
    const int iterations = args.error().empty() ? args.integer("iterations") : 0;
    if (!args.error().empty() || iterations <= 0) {
        std::cerr << (args.error().empty() ? "non-positive --iterations" : args.error()) << "\n"
                  << "Specify --scene, --output and positive --iterations.\n";
        return 1;
    }
    const std::string scene_dir = args.str("scene"), output_dir = args.str("output");
    const int downscale = std::max(1, args.integer("downscale"));

    auto t0 = std::chrono::steady_clock::now();
    std::cout << "Reading scene: " << scene_dir << std::endl;
    gs_native::ColmapScene colmap;
    if (!gs_native::ReadColmapScene(scene_dir, downscale, colmap)) {
        std::cerr << "Reading the COLMAP scene failed.\n";
        return 1;
    }
    std::cout << "Scene read: " << Seconds(t0) << " s" << std::endl;

    t0 = std::chrono::steady_clock::now();
    std::cout << "Initializing Gaussians..." << std::endl;
    gs_native::TrainingScene scene;
    scene.train_cameras = colmap.train_cameras;
    for (const auto& image : colmap.train_images) scene.train_images.push_back(image.rgb.data());
    scene.point_positions = colmap.point_positions.data();
    scene.point_colors = colmap.point_colors.data();
    scene.point_count = static_cast<int>(colmap.point_positions.size() / 3);
    gs_native::TrainingOptions options;
    options.bf16_sh = args.flag("precision");
    options.graph = args.flag("graph");
    options.max_gaussians = std::max(0, args.integer("max_gaussians"));
    options.exact_culling = args.flag("culled");
    options.sparse_adam = options.spatial_order = args.flag("sparse");
    options.fast_blend = args.flag("fast");
    options.fp32_ssim = args.flag("fp32_ssim");
    gs_native::GaussianSplatting gs;
    if (!gs.Initialize(scene, options)) {
        std::cerr << "Initialization failed.\n";
        return 1;
    }
    if (args.str("resume") != "none" && !gs.LoadCheckpoint(args.str("resume"))) {
        std::cerr << "Resuming from " << args.str("resume") << " failed.\n";
        return 1;
    }
    cudaDeviceSynchronize();
    std::cout << "Initialization: " << Seconds(t0) << " s" << std::endl;
    const int remaining = iterations - gs.GetCompleted();
    std::cout << "Cameras: " << scene.train_cameras.size() << ", initial Gaussians: " << scene.point_count
              << ", completed: " << gs.GetCompleted() << ", single-view updates: " << std::max(remaining, 0)
              << std::endl;

    t0 = std::chrono::steady_clock::now();
    if (remaining > 0 && !gs.Train(remaining)) {
        std::cerr << "Training failed.\n";
        return 1;
    }
    cudaDeviceSynchronize();
    const double total = Seconds(t0);
    std::cout << "Training total: " << total << " s, average: " << 1000.0 * total / std::max(remaining, 1)
              << " ms/update, Gaussians: " << gs.GetGaussians().gaussian_count_ << std::endl;
    if (args.str("checkpoint") != "none" && !gs.SaveCheckpoint(args.str("checkpoint"))) {
        std::cerr << "Saving the checkpoint failed.\n";
        return 1;
    }

    const std::filesystem::path model_dir = std::filesystem::absolute(output_dir);
    const std::filesystem::path cloud_dir = model_dir / "point_cloud" / ("iteration_" + std::to_string(iterations));
    std::filesystem::create_directories(cloud_dir);
    t0 = std::chrono::steady_clock::now();
    std::cout << "Saving model..." << std::endl;
    if (!gs.Save((cloud_dir / "point_cloud.ply").string())) {
        std::cerr << "Saving model failed.\n";
        return 1;
    }
    std::ofstream config(model_dir / "cfg_args");
    config << "Namespace(sh_degree=" << std::min(3, iterations / 1000)
           << ", source_path=" << std::quoted(std::filesystem::absolute(scene_dir).generic_string(), '\'')
           << ", model_path=" << std::quoted(model_dir.generic_string(), '\'') << ", images='images', resolution="
           << downscale << ", white_background=False, data_device='cuda', eval=True)\n";
    config.close();
    if (!config) {
        std::cerr << "Saving viewer configuration failed.\n";
        return 1;
    }
    std::cout << "Saving: " << Seconds(t0) << " s\nModel: " << (cloud_dir / "point_cloud.ply").string() << std::endl;
    return 0;
}
