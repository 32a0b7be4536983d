// Multi-view forward rendering: the tiles of many views (uneven resolutions)
// blended by one persistent launch, with the tile shape and threads per tile as
// template parameters (the autotuner's sweep), and the record-ordering kernels
// of the full-key sorts (48 / 64-bit tile|depth keys).
//
// Persistent kernel: CTAs take (view, tile) work items from a device counter,
// so views of different sizes share the machine without a launch per view and
// the tail of one view overlaps the next. The per-tile blend is the plain
// renderer's (front-to-back, conservative alpha-box culling per warp strip, the
// alpha floor before expf, early stop when the tile is saturated) with the
// same per-pixel arithmetic (renderer.cu:273-338), generalised to TW x TH tiles
// and THREADS threads: warp w owns a strip of TH / warps rows, lane l the
// column l % TW and the rows (l / TW) + p * (32 / TW) of that strip.
#include <algorithm>

#include "raster_common.cuh"
#include "kernels.h"
#include "multiview.h"

namespace gsn {

namespace {

constexpr int kBatch = 128;  // records staged per round

template <int TW, int TH, int THREADS>
struct Geometry {
    static constexpr int kWarps = THREADS / 32;
    static constexpr int kStripRows = TH / kWarps;       // rows per warp
    static constexpr int kRowsPerPass = 32 / TW;         // rows covered by one warp-wide pixel set
    static constexpr int kPix = kStripRows / kRowsPerPass;  // pixels per thread
    static_assert(kPix >= 1 && kStripRows % kRowsPerPass == 0, "tile shape / threads combination");
};

template <int TW, int TH, int THREADS>
__device__ __forceinline__ void blend_tile(const MultiView& v, int tile, float2* s_mean, float4* s_conic,
                                           float3* s_color, float4* s_box, float* s_floor) {
    using G = Geometry<TW, TH, THREADS>;
    constexpr int P = G::kPix;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int tx = tile % v.tiles_x, ty = tile / v.tiles_x;
    const int px = tx * TW + lane % TW;
    const int row0 = ty * TH + warp * G::kStripRows + lane / TW;
    const float fx = static_cast<float>(px);
    const float sx0 = static_cast<float>(tx * TW), sx1 = sx0 + (TW - 1);
    const float sy0 = static_cast<float>(ty * TH + warp * G::kStripRows), sy1 = sy0 + (G::kStripRows - 1);
    float fy[P], T[P];
    float3 C[P];
    bool done[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int py = row0 + p * G::kRowsPerPass;
        fy[p] = static_cast<float>(py);
        done[p] = !(px < v.width && py < v.height);
        T[p] = 1.0f;
        C[p] = make_float3(0.f, 0.f, 0.f);
    }
    const int64_t begin = v.tile_offsets[tile];
    const int64_t end = v.tile_offsets[tile + 1];
    for (int64_t base = begin; base < end; base += kBatch) {
        bool mine = true;
#pragma unroll
        for (int p = 0; p < P; ++p) mine = mine && done[p];
        if (__syncthreads_and(mine)) break;
        for (int slot = t; slot < kBatch; slot += THREADS) {
            const int64_t r = base + slot;
            float2 mean = make_float2(0.f, 0.f);
            float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
            float3 c = make_float3(0.f, 0.f, 0.f);
            if (r < end) {
                const uint32_t id = __ldg(v.tile_ids + r);
                mean = __ldg(v.means + id);
                q = __ldg(v.conic_opacity + id);
                const float* cp = reinterpret_cast<const float*>(v.colors) + 3ull * id;
                c = make_float3(__ldg(cp), __ldg(cp + 1), __ldg(cp + 2));
            }
            s_mean[slot] = mean;
            s_conic[slot] = q;
            s_color[slot] = c;
            s_box[slot] = alpha_box(mean, q);
            s_floor[slot] = alpha_floor(q.w);
        }
        __syncthreads();
        const int batch = static_cast<int>(min(static_cast<int64_t>(kBatch), end - base));
#pragma unroll 1
        for (int k = 0; k < kBatch / 32; ++k) {
            const int jl = k * 32 + lane;
            uint32_t m = __ballot_sync(0xffffffffu, jl < batch && box_hits(s_box[jl], sx0, sx1, sy0, sy1));
            while (m) {
                bool all = true;
#pragma unroll
                for (int p = 0; p < P; ++p) all = all && done[p];
                if (all) break;
                const int j = k * 32 + __ffs(m) - 1;
                m &= m - 1;
                const float2 mu = s_mean[j];
                const float4 q = s_conic[j];
                const float lim = s_floor[j];
                const float3 c = s_color[j];
                const float dx = mu.x - fx;
                float pw[P];
                bool act[P];
                bool any = false;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const float dy = mu.y - fy[p];
                    pw[p] = -0.5f * (q.x * dx * dx + q.z * dy * dy) - q.y * dx * dy;
                    act[p] = !done[p] && !(pw[p] > 0.0f) && !(pw[p] < lim);
                    any |= act[p];
                }
                if (!any) continue;
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    const float alpha = fminf(kAlphaMax, q.w * expf(pw[p]));
                    bool take = act[p] && !(alpha < kAlphaMin);
                    const float nextT = T[p] * (1.0f - alpha);
                    const bool stop = take && nextT < kTransmittanceMin;
                    done[p] = done[p] || stop;
                    take = take && !stop;
                    const float w = alpha * T[p];
                    C[p].x = take ? C[p].x + c.x * w : C[p].x;
                    C[p].y = take ? C[p].y + c.y * w : C[p].y;
                    C[p].z = take ? C[p].z + c.z * w : C[p].z;
                    T[p] = take ? nextT : T[p];
                }
            }
        }
        __syncthreads();  // staging of the next round overwrites this one
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
        const int py = row0 + p * G::kRowsPerPass;
        if (!(px < v.width && py < v.height)) continue;
        float* out = v.image + (static_cast<int64_t>(py) * v.width + px) * 3;
        out[0] = C[p].x + T[p] * v.background.x;
        out[1] = C[p].y + T[p] * v.background.y;
        out[2] = C[p].z + T[p] * v.background.z;
    }
}

template <int TW, int TH, int THREADS>
__global__ void __launch_bounds__(THREADS) multiview_kernel(MultiViewArgs a) {
    __shared__ float2 s_mean[kBatch];
    __shared__ float4 s_conic[kBatch];
    __shared__ float3 s_color[kBatch];
    __shared__ float4 s_box[kBatch];
    __shared__ float s_floor[kBatch];
    __shared__ int s_item;
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(a.queue, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= a.total_tiles) break;
        int v = 0;
        while (v + 1 < a.view_count && a.tile_prefix[v + 1] <= item) ++v;
        blend_tile<TW, TH, THREADS>(a.views[v], item - a.tile_prefix[v], s_mean, s_conic, s_color, s_box, s_floor);
    }
}

// Records in Gaussian-id order with a depth key per record (full-key orders).
__global__ void emit_keyed_kernel(const int* __restrict__ record_start, const int4* __restrict__ rects,
                                  const int* __restrict__ tile_counts, const uint32_t* __restrict__ depth_bits, int n,
                                  int tiles_x, int64_t capacity, uint32_t* __restrict__ tile_keys,
                                  uint32_t* __restrict__ depth_keys, uint32_t* __restrict__ ids) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || tile_counts[i] == 0) return;
    const int4 r = rects[i];
    int64_t o = record_start[i];
    for (int y = r.y; y < r.w; ++y)
        for (int x = r.x; x < r.z; ++x) {
            if (o >= capacity) return;
            tile_keys[o] = static_cast<uint32_t>(y * tiles_x + x);
            depth_keys[o] = depth_bits[i];
            ids[o] = static_cast<uint32_t>(i);
            ++o;
        }
}

__global__ void gather_records_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ tile_keys,
                                      const uint32_t* __restrict__ ids, int64_t count, uint32_t* __restrict__ tiles_out,
                                      uint32_t* __restrict__ ids_out) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const uint32_t r = order[p];
    tiles_out[p] = tile_keys[r];
    ids_out[p] = ids[r];
}

template <int TW, int TH, int THREADS>
int launch_multiview_config(const MultiViewArgs& a, int sms, cudaStream_t stream) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, multiview_kernel<TW, TH, THREADS>, THREADS, 0) !=
            cudaSuccess ||
        per_sm <= 0)
        return GSN_ERR_CUDA;
    const int grid = std::min(sms * per_sm, std::max(a.total_tiles, 1));
    multiview_kernel<TW, TH, THREADS><<<grid, THREADS, 0, stream>>>(a);
    return launched(1);
}

}  // namespace

bool multiview_config_valid(int tile_w, int tile_h, int threads) {
    if (!((tile_w == 16 && (tile_h == 16 || tile_h == 8)) || (tile_w == 8 && tile_h == 8))) return false;
    if (threads != 64 && threads != 128 && threads != 256) return false;
    const int warps = threads / 32, strip = tile_h / warps, rows_per_pass = 32 / tile_w;
    return strip >= rows_per_pass && strip % rows_per_pass == 0;
}

int launch_multiview(const MultiViewArgs& a, int tile_w, int tile_h, int threads, cudaStream_t stream) {
    if (a.total_tiles <= 0) return GSN_OK;
    if (!multiview_config_valid(tile_w, tile_h, threads)) return GSN_ERR_INVALID_ARGUMENT;
    static int sms[64] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return GSN_ERR_CUDA;
    if (!sms[device] && cudaDeviceGetAttribute(&sms[device], cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return GSN_ERR_CUDA;
    const int s = sms[device];
    if (tile_w == 16 && tile_h == 16) {
        if (threads == 64) return launch_multiview_config<16, 16, 64>(a, s, stream);
        if (threads == 128) return launch_multiview_config<16, 16, 128>(a, s, stream);
        return launch_multiview_config<16, 16, 256>(a, s, stream);
    }
    if (tile_w == 16 && tile_h == 8) {
        if (threads == 64) return launch_multiview_config<16, 8, 64>(a, s, stream);
        return launch_multiview_config<16, 8, 128>(a, s, stream);
    }
    return launch_multiview_config<8, 8, 64>(a, s, stream);
}

int launch_emit_keyed(const int* record_start, const int4* rects, const int* tile_counts, const uint32_t* depth_bits,
                      int n, int tiles_x, int64_t capacity, uint32_t* tile_keys, uint32_t* depth_keys, uint32_t* ids,
                      cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    emit_keyed_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(record_start, rects, tile_counts, depth_bits, n, tiles_x,
                                                            capacity, tile_keys, depth_keys, ids);
    return launched(1);
}

int launch_gather_records(const uint32_t* order, const uint32_t* tile_keys, const uint32_t* ids, int64_t count,
                          uint32_t* tiles_out, uint32_t* ids_out, cudaStream_t stream) {
    if (count <= 0) return GSN_OK;
    gather_records_kernel<<<ceil_div(count, 256), 256, 0, stream>>>(order, tile_keys, ids, count, tiles_out,
                                                                    ids_out);
    return launched(1);
}

}  // namespace gsn
