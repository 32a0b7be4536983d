/*
 * gsn_types.h - plain-C types shared by the gs-native B200 C ABI (gsn.h) and the
 * C++ drop-in layer.
 *
 * The layouts below are byte-compatible with the reference's device ABI in
 * src/core/types/buffers.h:10-33 (parameter row indices, CameraParams,
 * GaussianBuffers), so a caller that fills a gs_native::CameraParams can hand the
 * same bytes to any gsn_* entry point.
 */
#ifndef GSN_TYPES_H
#define GSN_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Row indices of the 58 x N structure-of-arrays parameter block (row stride == N).
 * Reference: src/core/types/buffers.h:10-15. SH coefficient k of colour channel c
 * lives in row GSN_SH_INDEX + c * 16 + k. */
enum {
    GSN_POSITION_INDEX = 0,
    GSN_LOG_SCALE_INDEX = 3,
    GSN_ROTATION_INDEX = 6,
    GSN_OPACITY_INDEX = 9,
    GSN_SH_INDEX = 10,
    GSN_PARAM_COUNT = 58,
    GSN_SH_COEFFS = 16,
    GSN_TILE_SIZE = 16
};

/* Pinhole camera, world->camera rotation R_c_w (row-major) and translation t_c_w.
 * Same member order and types as gs_native::CameraParams (buffers.h:17-28). */
typedef struct gsn_camera {
    float fx, fy, cx, cy;
    float R_c_w[9];
    float t_c_w[3];
    float near_depth, far_depth;
    int width, height;
    int64_t pixel_offset;
    int tile_count_x, tile_count_y;
    int tile_offset;
} gsn_camera;

/* Status codes returned by every gsn_* entry point (0 = success). */
enum {
    GSN_OK = 0,
    GSN_ERR_INVALID_ARGUMENT = -1,
    GSN_ERR_CUDA = -2,
    GSN_ERR_OUT_OF_MEMORY = -3,
    GSN_ERR_CAPACITY = -4,
    GSN_ERR_NOT_READY = -5,
    GSN_ERR_IO = -6,
    GSN_ERR_TIMEOUT = -7
};

#ifdef __cplusplus
}
#endif

#endif /* GSN_TYPES_H */
