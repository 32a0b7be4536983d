// (c) Per-tile front-to-back alpha blending.
//
// One 64-thread CTA per 16x16 tile, four pixels per thread, warp w owning the
// 16x8 pixel strip of rows 8w..8w+7 (raster_common.cuh). The tile's sorted
// records are staged into shared memory in batches of 128; while a batch is
// blended every thread already holds its two slots of the next batch in
// registers, so the id -> record gather overlaps the blend. Each record read from
// shared memory serves the thread's four pixels.
//
// Per batch each warp tests the records against its strip (conservative
// alpha >= 1/255 box) with four ballots and walks only the set bits, in order;
// per pixel, powers below the record's alpha floor are rejected before expf.
// Both tests only drop evaluations the exact per-pixel test would have skipped,
// so the result is unchanged. A CTA stops as soon as all of its pixels are
// saturated.
//
// The exact form evaluates the per-pixel arithmetic (power, alpha clamp at
// 0.99, the 1/255 skip and the 1e-4 transmittance stop) exactly as the
// reference does (renderer.cu:273-338), so images are bit-identical for
// identical inputs. The fast form takes alpha as ex2 of the power in log2
// units with the opacity folded in (raster_common.cuh fast_record: two FMAs and
// one MUFU per pixel, one compare for the 1/255 test) and updates the
// transmittance as T - alpha T; every pixel is evaluated branch-free. Besides the
// image the kernel records, per pixel, how many records were consumed up to its
// last contribution; the backward pass takes its replay's take set from it.
// A counting variant (RasterForwardArgs::pair_count) also sums the pairs taken.
#include "raster_common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

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

template <bool kFast, bool kCount>
__global__ void __launch_bounds__(kRasterThreads) raster_forward_kernel(RasterForwardArgs a) {
    pdl_begin();
    __shared__ float2 s_mean[kRasterBatch];
    __shared__ float4 s_conic[kRasterBatch];  // exact form: conic + opacity; fast form: fast_record terms
    __shared__ float3 s_color[kRasterBatch];
    __shared__ float4 s_box[kRasterBatch];
    __shared__ float s_floor[kRasterBatch];

    const int t = threadIdx.x;
    const int lane = t & 31;
    const int warp = t >> 5;
    const TileGeometry g = tile_geometry(a.cam);
    const float fx = static_cast<float>(g.px);
    float fy[kPixPerThread];
    bool done[kPixPerThread];
    float T[kPixPerThread];
    float3 C[kPixPerThread];
    int consumed[kPixPerThread];
    unsigned int pairs = 0;  // kCount: pairs this thread's pixels took
#pragma unroll
    for (int p = 0; p < kPixPerThread; ++p) {
        fy[p] = static_cast<float>(g.py[p]);
        done[p] = !(g.px < a.cam.width && g.py[p] < a.cam.height);
        T[p] = 1.0f;
        C[p] = make_float3(0.f, 0.f, 0.f);
        consumed[p] = 0;
    }

    const int64_t begin = a.tile_offsets[g.tile];
    const int64_t end = a.tile_offsets[g.tile + 1];

    Staged n0 = fetch(a, begin + t, end);
    Staged n1 = fetch(a, begin + t + kRasterThreads, end);
    for (int64_t base = begin; base < end; base += kRasterBatch) {
        const bool mine = done[0] && done[1] && done[2] && done[3];
        if (__syncthreads_and(mine)) break;
        s_mean[t] = n0.mean;
        s_conic[t] = kFast ? fast_record(n0.conic) : n0.conic;
        s_color[t] = n0.color;
        s_box[t] = alpha_box(n0.mean, n0.conic);
        if (!kFast) s_floor[t] = alpha_floor(n0.conic.w);
        s_mean[t + kRasterThreads] = n1.mean;
        s_conic[t + kRasterThreads] = kFast ? fast_record(n1.conic) : n1.conic;
        s_color[t + kRasterThreads] = n1.color;
        s_box[t + kRasterThreads] = alpha_box(n1.mean, n1.conic);
        if (!kFast) s_floor[t + kRasterThreads] = alpha_floor(n1.conic.w);
        __syncthreads();
        n0 = fetch(a, base + kRasterBatch + t, end);
        n1 = fetch(a, base + kRasterBatch + kRasterThreads + t, end);
        const int batch = static_cast<int>(min(static_cast<int64_t>(kRasterBatch), end - base));
        const int rel = static_cast<int>(base - begin);
        uint32_t* plane = a.record_warps ? a.record_warps + warp * a.record_words : nullptr;
#pragma unroll 1
        for (int k = 0; k < kRasterBatch / 32; ++k) {
            const int jl = k * 32 + lane;
            uint32_t m = __ballot_sync(0xffffffffu, jl < batch && box_hits(s_box[jl], g.sx0, g.sx1, g.sy0, g.sy1));
            uint32_t took = 0;  // records of this chunk a pixel of this lane took
            while (m && !(done[0] && done[1] && done[2] && done[3])) {
                const int j = k * 32 + __ffs(m) - 1;
                m &= m - 1;
                const float2 mu = s_mean[j];
                const float4 q = s_conic[j];
                const float3 c = s_color[j];
                const float dx = mu.x - fx;
                if constexpr (kFast) {
                    // fast_record terms (raster_common.cuh), the same expressions as
                    // the fast backward; every pixel evaluated branch-free, a pixel
                    // that does not take the record gets alpha = 0. Scalar
                    // arithmetic: this loop is bound by the ALU pipe, which the
                    // register moves of packed pairs would load further.
                    const float Ax = fmaf(q.x * dx, dx, q.w), Bx = q.y * dx;
                    const int consumed_if = rel + j + 1;
                    bool any = false;
#pragma unroll
                    for (int p = 0; p < kPixPerThread; ++p) {
                        const float dy = mu.y - fy[p];
                        const float pw2 = fmaf(fmaf(q.z, dy, Bx), dy, Ax);
                        const bool take = !done[p] && pw2 >= kLog2AlphaMin;
                        const float alpha = take ? fminf(kAlphaMax, ex2_approx(pw2)) : 0.0f;
                        float w = alpha * T[p];
                        // a live pixel's T stays >= 1e-4, so only a taken record can
                        // stop it, and a pixel that was already done has w = 0: the
                        // updated done flag alone decides whether w counts
                        done[p] = done[p] || T[p] - w < kTransmittanceMin;
                        w = done[p] ? 0.0f : w;
                        C[p].x = fmaf(c.x, w, C[p].x);
                        C[p].y = fmaf(c.y, w, C[p].y);
                        C[p].z = fmaf(c.z, w, C[p].z);
                        T[p] -= w;  // T (1 - alpha) as T - alpha T; unchanged at the stop
                        // alpha >= 1/255 and T >= 1e-4 make a taken record's w > 0
                        const bool took_p = w > 0.0f;
                        consumed[p] = took_p ? consumed_if : consumed[p];
                        any |= took_p;
                        if (kCount) pairs += took_p ? 1u : 0u;
                    }
                    took |= any ? 1u << (j & 31) : 0u;
                } else {
                    const float lim = s_floor[j];
                    const Power<false> power(q, dx);
                    // the four pixels are evaluated without branches (selects only),
                    // so their dependency chains interleave; values of a pixel that
                    // does not take the record are computed but discarded
                    float pw[kPixPerThread];
                    bool act[kPixPerThread];
                    bool any = false;
#pragma unroll
                    for (int p = 0; p < kPixPerThread; ++p) {
                        float dy = mu.y - fy[p];
                        pw[p] = power.at(dy);
                        act[p] = !done[p] && !(pw[p] > 0.0f) && !(pw[p] < lim);
                        any |= act[p];
                    }
                    if (!any) continue;
#pragma unroll
                    for (int p = 0; p < kPixPerThread; ++p) {
                        float alpha = fminf(kAlphaMax, gaussian_weight<false>(q.w, pw[p]));
                        bool take = act[p] && !(alpha < kAlphaMin);
                        float nextT = T[p] * (1.0f - alpha);
                        bool stop = take && nextT < kTransmittanceMin;
                        done[p] = done[p] || stop;
                        take = take && !stop;
                        float w = alpha * T[p];
                        C[p].x = take ? C[p].x + c.x * w : C[p].x;
                        C[p].y = take ? C[p].y + c.y * w : C[p].y;
                        C[p].z = take ? C[p].z + c.z * w : C[p].z;
                        T[p] = take ? nextT : T[p];
                        consumed[p] = take ? rel + j + 1 : consumed[p];
                        took |= take ? 1u << (j & 31) : 0u;
                        if (kCount) pairs += take ? 1u : 0u;
                    }
                }
            }
            if (plane) {
                // this warp strip's took-flags of the chunk's 32 records, one bit
                // each, into the plane at the records' global positions
#pragma unroll
                for (int o = 16; o; o >>= 1) took |= __shfl_xor_sync(0xffffffffu, took, o);
                if (lane == 0 && took) {
                    const int64_t r0 = base + k * 32;
                    const int off = static_cast<int>(r0 & 31);
                    atomicOr(plane + (r0 >> 5), took << off);
                    if (off) atomicOr(plane + (r0 >> 5) + 1, took >> (32 - off));
                }
            }
        }
    }
    if (kCount) {
        const unsigned long long warp_pairs = __reduce_add_sync(0xffffffffu, pairs);
        if (lane == 0 && warp_pairs) atomicAdd(a.pair_count, warp_pairs);
    }
#pragma unroll
    for (int p = 0; p < kPixPerThread; ++p) {
        if (!(g.px < a.cam.width && g.py[p] < a.cam.height)) continue;
        const int64_t pix = static_cast<int64_t>(g.py[p]) * a.cam.width + g.px;
        float* out = a.image + pix * 3;
        out[0] = C[p].x + T[p] * a.background.x;
        out[1] = C[p].y + T[p] * a.background.y;
        out[2] = C[p].z + T[p] * a.background.z;
        if (a.final_transmittance) a.final_transmittance[pix] = T[p];
        if (a.contributors) a.contributors[pix] = consumed[p];
    }
}

}  // namespace

int launch_raster_forward(const RasterForwardArgs& a, cudaStream_t stream) {
    int64_t tiles = static_cast<int64_t>(a.cam.tile_count_x) * a.cam.tile_count_y;
    if (tiles <= 0) return GSN_OK;
    const unsigned grid = static_cast<unsigned>(tiles);
    if (a.pair_count) {
        if (a.fast) launch_step(raster_forward_kernel<true, true>, grid, kRasterThreads, 0, stream, a);
        else launch_step(raster_forward_kernel<false, true>, grid, kRasterThreads, 0, stream, a);
    } else if (a.fast) {
        launch_step(raster_forward_kernel<true, false>, grid, kRasterThreads, 0, stream, a);
    } else {
        launch_step(raster_forward_kernel<false, false>, grid, kRasterThreads, 0, stream, a);
    }
    return launched(1);
}

}  // namespace gsn
