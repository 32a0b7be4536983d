// COLMAP scene reader without OpenCV (reference: src/io/data_io.cpp:79-418,
// ReadColmapScene). Reads sparse/0/{cameras,images,points3D}.bin (one PINHOLE
// camera, as the reference requires), images pre-decoded to binary PPM (P6) in
// images/ (for an image named "a.jpg" the file images/a.ppm is read; a name
// that already ends in .ppm is read as is), optional integer downscale by block
// averaging. Images are sorted by name; every 8th is a test view, the rest
// train views (data_io.cpp:372-381). Intrinsics are scaled to the image size
// with the reference's half-pixel shift (data_io.cpp:228-240).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "core/types/buffers.h"
#include "io/image.h"

namespace gs_native {

struct ColmapScene {
    std::vector<CameraParams> train_cameras, test_cameras;
    std::vector<ImageU8> train_images, test_images;
    std::vector<std::string> train_names, test_names;
    std::vector<float> point_positions;  // xyz
    std::vector<float> point_colors;     // rgb in [0, 1]
};

bool ReadColmapScene(const std::string& scene_dir, int downscale, ColmapScene& scene);

// Camera parameters of a view: near 0.2, far unbounded, 16x16 tiles.
CameraParams MakeCamera(int width, int height, float fx, float fy, float cx, float cy, const float R_c_w[9],
                        const float t_c_w[3]);

}  // namespace gs_native
