/*
 * gsn.h - C ABI of the gs-native B200 3D Gaussian Splatting training hot path.
 *
 * Plain C: pointers, sizes and opaque handles only. Every entry point returns a
 * gsn status (0 = GSN_OK, negative = error, see gsn_types.h) and never throws.
 * Device pointers are CUDA device addresses; `stream` is a cudaStream_t passed as
 * void* (NULL = legacy default stream). Invalid arguments return
 * GSN_ERR_INVALID_ARGUMENT without side effects, like the reference's `false`
 * returns (e.g. renderer.cu:379-381, 451-454; density_controller.cu:473-481).
 *
 * The handle-based objects wrap the C++ drop-in classes of the gs_native
 * namespace (same semantics as the reference classes they replace); the
 * stateless stage functions expose single kernels for FFI callers and for the
 * parity tests.
 */
#ifndef GSN_H
#define GSN_H

#include <stddef.h>
#include <stdint.h>

#include "gsn_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ library */

/* Library version string. */
const char* gsn_version(void);

/* Synchronous byte copy between host/device memory (cudaMemcpyDefault). For FFI
 * callers without their own CUDA bindings. */
int gsn_memcpy(void* dst, const void* src, size_t bytes);

/* Blocks until all work on `stream` is done. */
int gsn_stream_synchronize(void* stream);

/* ------------------------------------------------------------------ renderer
 * Replaces gs_native::Renderer (reference src/core/render/renderer.h:10-89).
 */
typedef struct gsn_renderer gsn_renderer;

int gsn_renderer_create(gsn_renderer** out);
int gsn_renderer_destroy(gsn_renderer* r);
int gsn_renderer_set_stream(gsn_renderer* r, void* stream);

/* Renderer::Render (renderer.h:21-26; renderer.cu:359-372): project the 58 x count
 * SoA `params` (device), build the depth-ordered per-tile lists and blend into
 * `image` (device, fp32 HWC RGB, width*height*3). `background` is a host float[3].
 * sh_degree is clamped to [0, 3]. */
int gsn_renderer_render(gsn_renderer* r, const float* params, int count, const gsn_camera* camera,
                        const float* background, float* image, int sh_degree);

/* Device pointers owned by the renderer, valid until the next render call.
 * Getters of renderer.h:28-54 plus the extensions documented in renderer.h. */
typedef struct gsn_renderer_buffers {
    const float* means;            /* float2[count]: (u, v) */
    const float* conic_opacity;    /* float4[count]: (a, b, c, opacity) */
    const float* colors;           /* float3[count] */
    const float* depths;           /* float[count], valid where tile_counts > 0 */
    const int* rects;              /* int4[count]: tile rect [x0, y0, x1, y1), valid where tile_counts > 0 */
    const int* tile_counts;        /* int[count] */
    const float* radii;            /* float[count], 0 when culled */
    const int* tile_gaussian_ids;  /* int[record_count] sorted by (tile, depth, id) */
    const int64_t* tile_offsets;   /* int64[tiles + 1] */
    const int* contributors;       /* int[width * height]: records consumed per pixel */
    const int* record_count;       /* device int */
    const int* overflow;           /* device int, nonzero when a fixed capacity overflowed */
    int64_t record_count_host;     /* host copy (grow mode) */
    int gaussian_capacity;
    int tile_capacity;
} gsn_renderer_buffers;
int gsn_renderer_get_buffers(gsn_renderer* r, gsn_renderer_buffers* out);

/* Renderer::GetRecordOffsets (renderer.h:44-46): exclusive scan of tile counts in
 * id order, count + 1 entries. */
int gsn_renderer_record_offsets(gsn_renderer* r, const int** out);

/* Fixed record capacity (0 = grow on demand, the reference behaviour). */
int gsn_renderer_set_record_capacity(gsn_renderer* r, int64_t records);

#ifdef __cplusplus
}
#endif

#endif /* GSN_H */
