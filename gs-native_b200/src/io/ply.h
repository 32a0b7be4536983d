// Gaussian PLY export/import (reference: src/io/data_io.h:15-22,
// data_io.cpp:296-325, 420-590).
//
// Binary little-endian rows of 62 floats: x y z, nx ny nz (0), f_dc_0..2,
// f_rest_0..44 (channel-major), opacity (logit), scale_0..2 (log), rot_0..3
// (quaternion w, x, y, z from the axis-angle rotation). Reading accepts any
// float property order, requires every named property, rejects truncated files
// and non-finite values, and converts the quaternion back to axis-angle.
#pragma once

#include <string>
#include <vector>

namespace gs_native {

// Host Gaussian of the PLY IO (the fields of the reference's gs_native::Gaussian,
// gaussian.h:12-42, without Eigen): sh_[k][c] is coefficient k of channel c.
struct Gaussian {
    float position_[3] = {0, 0, 0};
    float log_scale_[3] = {0, 0, 0};
    float rotation_[3] = {0, 0, 0};
    float opacity_logit_ = 0.0f;
    float sh_[16][3] = {};
};

bool WriteGaussiansPly(const std::string& path, const std::vector<Gaussian>& gaussians);
bool ReadGaussiansPly(const std::string& path, std::vector<Gaussian>& gaussians);

// 58 x count SoA <-> host Gaussians.
std::vector<Gaussian> UnpackGaussians(const float* params, int count);
std::vector<float> PackGaussians(const std::vector<Gaussian>& gaussians);

}  // namespace gs_native
