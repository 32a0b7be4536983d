// Drop-in parameter layout and device views of gs_native (reference:
// src/core/types/buffers.h:10-58). Field order, types and sizes are kept
// identical because these structs are the ABI between the caller and the stage
// classes; CameraParams is byte-compatible with gsn_camera of the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "gsn_types.h"

namespace gs_native {

constexpr int kPositionIndex = GSN_POSITION_INDEX;
constexpr int kLogScaleIndex = GSN_LOG_SCALE_INDEX;
constexpr int kRotationIndex = GSN_ROTATION_INDEX;
constexpr int kOpacityIndex = GSN_OPACITY_INDEX;
constexpr int kShIndex = GSN_SH_INDEX;
constexpr int kMaxParamCount = GSN_PARAM_COUNT;

struct CameraParams {
    float fx_, fy_, cx_, cy_;
    float R_c_w_[9];
    float t_c_w_[3];
    float near_depth_, far_depth_;

    int width_, height_;
    int64_t pixel_offset_;

    int tile_count_x_, tile_count_y_;
    int tile_offset_;
};

static_assert(sizeof(CameraParams) == sizeof(gsn_camera), "CameraParams must match gsn_camera");
static_assert(offsetof(CameraParams, pixel_offset_) == offsetof(gsn_camera, pixel_offset),
              "CameraParams must match gsn_camera");
static_assert(offsetof(CameraParams, tile_offset_) == offsetof(gsn_camera, tile_offset),
              "CameraParams must match gsn_camera");

inline const gsn_camera& AsGsnCamera(const CameraParams& c) {
    return *reinterpret_cast<const gsn_camera*>(&c);
}

// Non-owning view of a 58 x N SoA parameter block (row stride == count).
struct GaussianBuffers {
    float* gaussians_ = nullptr;
    int gaussian_count_ = 0;
};

struct ViewBuffers {
    CameraParams* cameras_ = nullptr;
    int camera_count_ = 0;
    int tile_count_ = 0;
    uint8_t* images_ = nullptr;
};

struct TileListBuffers {
    int* gaussian_ids_ = nullptr;
    float* gaussian_depths_ = nullptr;
    int* gaussian_counts_ = nullptr;
    int64_t* gaussian_offsets_ = nullptr;
    int64_t capacity_ = 0;
};

}  // namespace gs_native
