// (d) Analytic backward of the per-tile blend.
//
// One CTA per 16x16 tile, one thread per pixel, replaying the tile's records
// front to back against the pixel's final colour like the reference
// (solver.cu:325-466), with three changes that leave the per-pair arithmetic
// untouched:
//   * the replay of a tile stops at the largest per-pixel contributor count the
//     forward pass recorded, and a pixel stops at its own count, so records
//     behind the saturation point are never re-evaluated;
//   * the 11 per-pair values of a warp are combined with a butterfly
//     reduce-scatter (13 shuffles instead of 55): after five halving steps lane
//     pairs hold the warp sum of one value each;
//   * warp sums are accumulated per batch in shared memory (shared-memory
//     float atomics) and flushed with one global atomic per (Gaussian, value)
//     and tile, instead of one per warp.
// Per-Gaussian output (12 floats, Gaussian-major): d(u, v), d(cov a, b, c),
// d(opacity logit), d(r, g, b), sum|du|, sum|dv|, 0.
#include "common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

constexpr int kBatch = 256;
constexpr int kVals = 12;

struct Rec {
    float2 mean;
    float4 conic;
    float3 color;
};

__device__ __forceinline__ float sel(bool c, float a, float b) { return c ? a : b; }

__global__ void __launch_bounds__(kTilePixels) raster_backward_kernel(RasterBackwardArgs a) {
    __shared__ uint32_t s_id[kBatch];
    __shared__ float2 s_mean[kBatch];
    __shared__ float4 s_conic[kBatch];
    __shared__ float3 s_color[kBatch];
    __shared__ float s_acc[kBatch * kVals];
    __shared__ int s_bound;

    const int t = threadIdx.x;
    const int lane = t & 31;
    const int tile = blockIdx.x;
    const int tx = tile % a.cam.tile_count_x;
    const int ty = tile / a.cam.tile_count_x;
    const int px = tx * kTile + (t % kTile);
    const int py = ty * kTile + (t / kTile);
    const bool inside = px < a.cam.width && py < a.cam.height;
    const float fx = static_cast<float>(px), fy = static_cast<float>(py);
    const int64_t pix = static_cast<int64_t>(py) * a.cam.width + px;

    const int64_t begin = a.tile_offsets[tile];
    const int64_t end_all = a.tile_offsets[tile + 1];
    float fin[3] = {0.f, 0.f, 0.f}, gI[3] = {0.f, 0.f, 0.f}, prefix[3] = {0.f, 0.f, 0.f};
    int limit = 0;
    if (inside) {
        for (int c = 0; c < 3; ++c) {
            fin[c] = a.image[pix * 3 + c];
            gI[c] = a.image_grad[pix * 3 + c];
        }
        limit = a.contributors ? a.contributors[pix] : static_cast<int>(end_all - begin);
    }
    if (t == 0) s_bound = 0;
    __syncthreads();
    {
        int wmax = __reduce_max_sync(0xffffffffu, limit);
        if (lane == 0 && wmax > 0) atomicMax(&s_bound, wmax);
    }
    __syncthreads();
    const int64_t end = begin + min(static_cast<int64_t>(s_bound), end_all - begin);
    bool done = !inside;
    float T = 1.0f;

    for (int64_t base = begin; base < end; base += kBatch) {
        const int batch = static_cast<int>(min(static_cast<int64_t>(kBatch), end - base));
        if (t < batch) {
            uint32_t id = __ldg(a.tile_ids + base + t);
            s_id[t] = id;
            s_mean[t] = __ldg(a.means + id);
            s_conic[t] = __ldg(a.conic_opacity + id);
            const float* c = reinterpret_cast<const float*>(a.colors) + 3ull * id;
            s_color[t] = make_float3(__ldg(c), __ldg(c + 1), __ldg(c + 2));
        }
        for (int k = t; k < kBatch * kVals; k += kTilePixels) s_acc[k] = 0.0f;
        __syncthreads();
        for (int j = 0; j < batch; ++j) {
            float v[kVals];
#pragma unroll
            for (int k = 0; k < kVals; ++k) v[k] = 0.0f;
            bool has = false;
            if (!done && static_cast<int>(base - begin) + j >= limit) done = true;
            if (!done) {
                float2 m = s_mean[j];
                float dx = m.x - fx, dy = m.y - fy;
                float4 q = s_conic[j];
                float power = -0.5f * (q.x * dx * dx + q.z * dy * dy) - q.y * dx * dy;
                if (power <= 0.0f) {
                    float raw = q.w * expf(power);
                    float alpha = fminf(kAlphaMax, raw);
                    if (alpha >= kAlphaMin) {
                        float nextT = T * (1.0f - alpha);
                        if (nextT < kTransmittanceMin) {
                            done = true;
                        } else {
                            has = true;
                            float3 col = s_color[j];
                            float cc[3] = {col.x, col.y, col.z};
                            float dalpha = 0.0f;
                            float w = alpha * T;
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                dalpha += gI[c] * (prefix[c] + T * cc[c] - fin[c]) / (1.0f - alpha);
                                v[6 + c] = w * gI[c];
                            }
                            if (raw < kAlphaMax) {
                                float common = dalpha * raw;
                                float qx = q.x * dx + q.y * dy;
                                float qy = q.y * dx + q.z * dy;
                                v[0] = -common * qx;
                                v[1] = -common * qy;
                                v[2] = 0.5f * common * qx * qx;
                                v[3] = common * qx * qy;
                                v[4] = 0.5f * common * qy * qy;
                                v[5] = common * (1.0f - q.w);
                            }
#pragma unroll
                            for (int c = 0; c < 3; ++c) prefix[c] += cc[c] * w;
                            T = nextT;
                        }
                    }
                }
            }
            v[9] = fabsf(v[0]);
            v[10] = fabsf(v[1]);
            if (__any_sync(0xffffffffu, has)) {
                // butterfly reduce-scatter of the 12 slots (slot 11 is padding)
                const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
                float k6[6];
#pragma unroll
                for (int i = 0; i < 6; ++i) {
                    float send = sel(b4, v[i], v[6 + i]);
                    k6[i] = sel(b4, v[6 + i], v[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
                }
                float k3[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    float send = sel(b3, k6[i], k6[3 + i]);
                    k3[i] = sel(b3, k6[3 + i], k6[i]) + __shfl_xor_sync(0xffffffffu, send, 8);
                }
                float k4[4] = {k3[0], k3[1], k3[2], 0.0f};
                float k2[2];
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    float send = sel(b2, k4[i], k4[2 + i]);
                    k2[i] = sel(b2, k4[2 + i], k4[i]) + __shfl_xor_sync(0xffffffffu, send, 4);
                }
                float send = sel(b1, k2[0], k2[1]);
                float k1 = sel(b1, k2[1], k2[0]) + __shfl_xor_sync(0xffffffffu, send, 2);
                k1 += __shfl_xor_sync(0xffffffffu, k1, 1);
                const int low = (b2 ? 2 : 0) + (b1 ? 1 : 0);
                const int field = (b4 ? 6 : 0) + (b3 ? 3 : 0) + low;
                if ((lane & 1) == 0 && low < 3 && field < 11 && k1 != 0.0f) atomicAdd(&s_acc[j * kVals + field], k1);
            }
        }
        __syncthreads();
        for (int k = t; k < batch * kVals; k += kTilePixels) {
            float val = s_acc[k];
            if (val != 0.0f) atomicAdd(a.grad_out + static_cast<int64_t>(s_id[k / kVals]) * kVals + k % kVals, val);
        }
        __syncthreads();
    }
}

}  // namespace

int launch_raster_backward(const RasterBackwardArgs& a, cudaStream_t stream) {
    int64_t tiles = static_cast<int64_t>(a.cam.tile_count_x) * a.cam.tile_count_y;
    if (tiles <= 0) return GSN_OK;
    raster_backward_kernel<<<static_cast<unsigned>(tiles), kTilePixels, 0, stream>>>(a);
    return launched(1);
}

}  // namespace gsn
