// (c) Per-tile front-to-back alpha blending.
//
// One CTA per 16x16 tile, one thread per pixel. The tile's sorted records are
// staged into shared memory in batches of 256; while a batch is blended, every
// thread already holds its slot of the next batch in registers (software
// pipelining of the id -> record gather), so the gather latency overlaps the
// blend. A CTA stops as soon as all of its pixels are saturated.
//
// The per-pixel arithmetic (power, alpha clamp at 0.99, the 1/255 skip and the
// 1e-4 transmittance stop) is evaluated exactly as the reference does
// (renderer.cu:273-338), so images are bit-identical for identical inputs.
// Besides the image the kernel records, per pixel, how many records were
// consumed before the pixel stopped contributing; the backward pass uses it to
// bound its replay.
#include "common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

constexpr int kBatch = 256;

struct Staged {
    float2 mean;
    float4 conic;
    float3 color;
};

__device__ __forceinline__ Staged fetch(const RasterForwardArgs& a, int64_t r, int64_t end) {
    Staged s;
    if (r < end) {
        uint32_t id = __ldg(a.tile_ids + r);
        s.mean = __ldg(a.means + id);
        s.conic = __ldg(a.conic_opacity + id);
        const float* c = reinterpret_cast<const float*>(a.colors) + 3ull * id;
        s.color = make_float3(__ldg(c), __ldg(c + 1), __ldg(c + 2));
    } else {
        s.mean = make_float2(0.f, 0.f);
        s.conic = make_float4(0.f, 0.f, 0.f, 0.f);
        s.color = make_float3(0.f, 0.f, 0.f);
    }
    return s;
}

__global__ void __launch_bounds__(kTilePixels) raster_forward_kernel(RasterForwardArgs a) {
    __shared__ float2 s_mean[kBatch];
    __shared__ float4 s_conic[kBatch];
    __shared__ float3 s_color[kBatch];

    const int t = threadIdx.x;
    const int tile = blockIdx.x;
    const int tx = tile % a.cam.tile_count_x;
    const int ty = tile / a.cam.tile_count_x;
    const int px = tx * kTile + (t % kTile);
    const int py = ty * kTile + (t / kTile);
    const bool inside = px < a.cam.width && py < a.cam.height;
    const float fx = static_cast<float>(px);
    const float fy = static_cast<float>(py);

    const int64_t begin = a.tile_offsets[tile];
    const int64_t end = a.tile_offsets[tile + 1];

    bool done = !inside;
    float T = 1.0f;
    float3 C = make_float3(0.f, 0.f, 0.f);
    int consumed = 0;  // 1 + index of the last contributing record

    Staged next = fetch(a, begin + t, end);
    for (int64_t base = begin; base < end; base += kBatch) {
        if (__syncthreads_count(done) == kTilePixels) break;
        s_mean[t] = next.mean;
        s_conic[t] = next.conic;
        s_color[t] = next.color;
        __syncthreads();
        next = fetch(a, base + kBatch + t, end);
        const int batch = static_cast<int>(min(static_cast<int64_t>(kBatch), end - base));
        for (int j = 0; !done && j < batch; ++j) {
            float dx = s_mean[j].x - fx;
            float dy = s_mean[j].y - fy;
            float4 q = s_conic[j];
            float power = -0.5f * (q.x * dx * dx + q.z * dy * dy) - q.y * dx * dy;
            if (power > 0.0f) continue;
            float alpha = fminf(kAlphaMax, q.w * expf(power));
            if (alpha < kAlphaMin) continue;
            float nextT = T * (1.0f - alpha);
            if (nextT < kTransmittanceMin) {
                done = true;
                continue;
            }
            float w = alpha * T;
            float3 c = s_color[j];
            C.x += c.x * w;
            C.y += c.y * w;
            C.z += c.z * w;
            T = nextT;
            consumed = static_cast<int>(base - begin) + j + 1;
        }
    }
    if (inside) {
        const int64_t pix = static_cast<int64_t>(py) * a.cam.width + px;
        float* out = a.image + pix * 3;
        out[0] = C.x + T * a.background.x;
        out[1] = C.y + T * a.background.y;
        out[2] = C.z + T * a.background.z;
        if (a.final_transmittance) a.final_transmittance[pix] = T;
        if (a.contributors) a.contributors[pix] = consumed;
    }
}

}  // namespace

int launch_raster_forward(const RasterForwardArgs& a, cudaStream_t stream) {
    int64_t tiles = static_cast<int64_t>(a.cam.tile_count_x) * a.cam.tile_count_y;
    if (tiles <= 0) return GSN_OK;
    raster_forward_kernel<<<static_cast<unsigned>(tiles), kTilePixels, 0, stream>>>(a);
    return launched(1);
}

}  // namespace gsn
