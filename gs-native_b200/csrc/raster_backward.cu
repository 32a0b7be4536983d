// (d) Analytic backward of the per-tile blend.
//
// One 64-thread CTA per 16x16 tile, four pixels per thread (raster_common.cuh),
// replaying the tile's records front to back against each pixel's final colour
// like the reference (solver.cu:325-466), with these changes:
//   * the take set is the forward pass's: records [0, limit) of a tile hold
//     every record a pixel took (limit = the per-pixel contributor count the
//     forward records), so a pixel takes record idx when idx < limit and the
//     per-pixel alpha test passes; the transmittance stop needs no replay, and
//     a warp stops at its pixels' largest limit, the CTA at its own;
//   * a thread sums the contributions of its four pixels in registers, so one
//     warp reduction serves 128 pixel-record pairs; the four pixels are
//     evaluated branch-free (a pixel that does not take a record gets
//     alpha = 0, which zeroes its terms), so their dependency chains interleave;
//   * the 11 per-pair values of a warp are combined with a butterfly
//     reduce-scatter (13 shuffles instead of 55): after five halving steps lane
//     pairs hold the warp sum of one value each;
//   * warp sums are accumulated per batch in shared memory (shared-memory
//     float atomics) and flushed with one 16-byte vector reduction per four
//     values of a Gaussian and tile (three per Gaussian) when grad_out is
//     16-byte aligned;
//   * each warp walks only the records that some pixel of its 16x8 strip took
//     in the forward pass (per-record strip flags the forward writes) and whose
//     conservative alpha >= 1/255 box reaches the strip;
//   * the colour term of dL/dalpha is carried per pixel as two scalars (the
//     gradient-weighted final colour and the gradient-weighted colour in front
//     of the record) instead of three channel sums; the fast form carries their
//     difference as one value;
//   * per-record factors leave the per-pixel loop: d(cov a) and d(cov c) are
//     accumulated without the power's factor 1/2 and d(opacity logit) without
//     the sigmoid's (1 - o), applied once per record before the reduction;
//   * the fast form evaluates alpha as ex2 of the power in log2 units with the
//     opacity folded in (two FMAs, one MUFU per pixel; raster_common.cuh
//     fast_record), takes a pixel on one compare and divides by (1 - alpha)
//     through the hardware reciprocal; the exact form keeps the reference's
//     power expression, expf and the correctly rounded reciprocal;
//   * the fast form runs pixels in pairs in packed FP32x2 arithmetic
//     (raster_common.cuh fma2/mul2/add2, one instruction per two operations;
//     the alpha test, clamp and MUFU operations stay per pixel); its
//     transmittance update T - alpha T is the fast forward's expression;
//   * with the forward's take flags (the renderer always passes them) the fast
//     form runs one warp per tile with eight pixels per lane
//     (raster_backward_tile_kernel): a record some pixel of the tile took
//     costs one visit - staging, column terms and butterfly reduction - where
//     a warp per strip pays them twice for a record both strips took, and
//     the reduced values are stored without atomics;
//   * at most 80 registers (12 CTAs, 24 warps per SM): the exact form uses 80,
//     the fast form 67.
// Per-Gaussian output (12 floats, Gaussian-major): d(u, v), d(cov a, b, c),
// d(opacity logit), d(r, g, b), sum|du|, sum|dv|, 0.
#include "raster_common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

constexpr int kVals = 12;

__device__ __forceinline__ float sel(bool c, float a, float b) { return c ? a : b; }

// Element-wise atomic add of four floats at a 16-byte aligned global address
// (PTX red.global.add with a .v4.f32 vector, sm_90 and later).
__device__ __forceinline__ void red_add_v4(float* address, float4 v) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(address), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}

template <bool kFast>
__global__ void __launch_bounds__(kRasterThreads, 12) raster_backward_kernel(RasterBackwardArgs a) {
    pdl_begin();
    __shared__ uint32_t s_id[kRasterBatch];
    __shared__ float2 s_mean[kRasterBatch];
    __shared__ float4 s_conic[kRasterBatch];
    __shared__ float4 s_fast[kRasterBatch];   // fast form: fast_record terms
    __shared__ float3 s_color[kRasterBatch];
    __shared__ float4 s_box[kRasterBatch];
    __shared__ float s_floor[kRasterBatch];   // exact form: alpha floor
    __shared__ uint16_t s_warps[kRasterBatch];
    __shared__ __align__(16) float s_acc[kRasterBatch * kVals];
    __shared__ int s_bound;

    const int t = threadIdx.x;
    const int lane = t & 31;
    const int warp_shift = 8 * (t >> 5);
    const TileGeometry g = tile_geometry(a.cam);
    const float fx = static_cast<float>(g.px);
    const int64_t begin = a.tile_offsets[g.tile];
    const int64_t end_all = a.tile_offsets[g.tile + 1];

    float fy[kPixPerThread], T[kPixPerThread];
    // per pixel: dL/dcolour, S = dL/dcolour . final colour and P = dL/dcolour .
    // colour accumulated in front of the current record (the fast form carries
    // P - S in P)
    float gI[kPixPerThread][3], S[kPixPerThread], P[kPixPerThread];
    // records [0, limit) of the tile hold every record the pixel took in the
    // forward pass; past it the pixel took nothing (its transmittance stop, or
    // the end of the list), so limit alone replays the forward's stop
    int limit[kPixPerThread];
    int my_bound = 0;
#pragma unroll
    for (int p = 0; p < kPixPerThread; ++p) {
        fy[p] = static_cast<float>(g.py[p]);
        T[p] = 1.0f;
        limit[p] = 0;
        const bool inside = g.px < a.cam.width && g.py[p] < a.cam.height;
        S[p] = P[p] = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) gI[p][c] = 0.0f;
        if (inside) {
            const int64_t pix = static_cast<int64_t>(g.py[p]) * a.cam.width + g.px;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                gI[p][c] = a.image_grad[pix * 3 + c];
                S[p] += gI[p][c] * a.image[pix * 3 + c];
            }
            limit[p] = a.contributors[pix];
        }
        my_bound = max(my_bound, limit[p]);
        if (kFast) P[p] = -S[p];
    }
    // fast form: the pixels as two packed pairs (2h, 2h + 1)
    float2 nfy2[2], T2[2], P2[2], gI2[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        nfy2[h] = make_float2(-fy[2 * h], -fy[2 * h + 1]);
        T2[h] = pk(1.0f);
        P2[h] = make_float2(P[2 * h], P[2 * h + 1]);
#pragma unroll
        for (int c = 0; c < 3; ++c) gI2[h][c] = make_float2(gI[2 * h][c], gI[2 * h + 1][c]);
    }
    // the warp's replay ends at its pixels' largest bound, the CTA's at its own
    const int warp_bound = __reduce_max_sync(0xffffffffu, my_bound);
    if (t == 0) s_bound = 0;
    __syncthreads();
    if (lane == 0 && warp_bound > 0) atomicMax(&s_bound, warp_bound);
    __syncthreads();
    const int64_t end = begin + min(static_cast<int64_t>(s_bound), end_all - begin);

    for (int64_t base = begin; base < end; base += kRasterBatch) {
        const int batch = static_cast<int>(min(static_cast<int64_t>(kRasterBatch), end - base));
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int slot = t + h * kRasterThreads;
            if (slot < batch) {
                uint32_t id = __ldg(a.tile_ids + base + slot);
                s_id[slot] = id;
                float2 mean = __ldg(a.means + id);
                float4 q = __ldg(a.conic_opacity + id);
                s_mean[slot] = mean;
                s_conic[slot] = q;
                const float* c = reinterpret_cast<const float*>(a.colors) + 3ull * id;
                s_color[slot] = make_float3(__ldg(c), __ldg(c + 1), __ldg(c + 2));
                // with the forward's take bits the box test is implied (a record
                // some strip pixel took reaches that strip); without them it runs
                if (!a.record_warps) s_box[slot] = alpha_box(mean, q);
                if (kFast) s_fast[slot] = fast_record(q);
                else s_floor[slot] = alpha_floor(q.w);
                uint16_t flags = 0x0101;
                if (a.record_warps) {
                    const int64_t r = base + slot;
                    const uint32_t bit = 1u << (r & 31);
                    flags = static_cast<uint16_t>(((a.record_warps[r >> 5] & bit) ? 0x0001 : 0) |
                                                  ((a.record_warps[a.record_words + (r >> 5)] & bit) ? 0x0100 : 0));
                }
                s_warps[slot] = flags;
            }
        }
        for (int k = t; k < kRasterBatch * kVals; k += kRasterThreads) s_acc[k] = 0.0f;
        __syncthreads();
        const int rel = static_cast<int>(base - begin);
        // this warp's records of the batch: those before its bound
        const int wend = min(batch, warp_bound - rel);
#pragma unroll 1
        for (int k = 0; k * 32 < wend; ++k) {
            const int jl = k * 32 + lane;
            // records the forward pass took somewhere in this warp's strip (every
            // other record leaves the strip's pixels unchanged)
            uint32_t m = __ballot_sync(0xffffffffu, jl < wend && ((s_warps[jl] >> warp_shift) & 1u) &&
                                                        (a.record_warps ||
                                                         box_hits(s_box[jl], g.sx0, g.sx1, g.sy0, g.sy1)));
            while (m) {
                const int j = k * 32 + __ffs(m) - 1;
                m &= m - 1;
                const int idx = rel + j;
                const float2 mu = s_mean[j];
                const float4 q = s_conic[j];
                const float3 col = s_color[j];
                const float cc[3] = {col.x, col.y, col.z};
                const float dx = mu.x - fx;
                const float qxdx = q.x * dx, qydx = q.y * dx;
                float v[kVals];
#pragma unroll
                for (int i = 0; i < kVals; ++i) v[i] = 0.0f;
                // four pixels evaluated without branches (selects only) so their
                // dependency chains interleave; a pixel that does not take the
                // record gets alpha = 0, which zeroes its contributions
                if constexpr (kFast) {
                    // the two pixel pairs in packed FP32x2 arithmetic; the alpha
                    // test, clamp and the MUFU operations stay per pixel
                    const float4 kf = s_fast[j];
                    const float Ax = fmaf(kf.x * dx, dx, kf.w), Bx = kf.y * dx;
                    const float2 m1 = pk(-1.0f), one = pk(1.0f);
                    float2 acc[9];
#pragma unroll
                    for (int i = 0; i < 9; ++i) acc[i] = pk(0.0f);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float2 dy = add2(pk(mu.y), nfy2[h]);
                        const float2 pw2 = fma2(fma2(pk(kf.z), dy, pk(Bx)), dy, pk(Ax));
                        const bool take0 = idx < limit[2 * h] && pw2.x >= kLog2AlphaMin;
                        const bool take1 = idx < limit[2 * h + 1] && pw2.y >= kLog2AlphaMin;
                        float2 alpha;
                        alpha.x = take0 ? fminf(kAlphaMax, ex2_approx(pw2.x)) : 0.0f;
                        alpha.y = take1 ? fminf(kAlphaMax, ex2_approx(pw2.y)) : 0.0f;
                        // d alpha / d power: raw below the clamp, 0 when clamped or not taken
                        const float2 r = make_float2(alpha.x < kAlphaMax ? alpha.x : 0.0f,
                                                     alpha.y < kAlphaMax ? alpha.y : 0.0f);
                        const float2 w = mul2(alpha, T2[h]);
                        const float2 om = fma2(alpha, m1, one);  // 1 - alpha
                        const float2 inv = make_float2(one_over<true>(om.x), one_over<true>(om.y));
                        float2 G = mul2(gI2[h][0], pk(cc[0]));
                        G = fma2(gI2[h][1], pk(cc[1]), G);
                        G = fma2(gI2[h][2], pk(cc[2]), G);
                        // dL/dalpha = (dL/dC . (colour in front + T c - final)) / (1 - alpha)
                        const float2 dalpha = mul2(fma2(T2[h], G, P2[h]), inv);
#pragma unroll
                        for (int c = 0; c < 3; ++c) acc[6 + c] = fma2(w, gI2[h][c], acc[6 + c]);
                        const float2 common = mul2(dalpha, r);
                        const float2 qx = fma2(pk(q.y), dy, pk(qxdx));
                        const float2 qy = fma2(pk(q.z), dy, pk(qydx));
                        const float2 cqx = mul2(common, qx), cqy = mul2(common, qy);
                        acc[0] = fma2(cqx, m1, acc[0]);
                        acc[1] = fma2(cqy, m1, acc[1]);
                        acc[2] = fma2(cqx, qx, acc[2]);  // halved once per record below
                        acc[3] = fma2(cqx, qy, acc[3]);
                        acc[4] = fma2(cqy, qy, acc[4]);  // halved once per record below
                        acc[5] = add2(acc[5], common);   // times (1 - o) once per record below
                        v[9] += fabsf(cqx.x) + fabsf(cqx.y);
                        v[10] += fabsf(cqy.x) + fabsf(cqy.y);
                        P2[h] = fma2(w, G, P2[h]);
                        // T (1 - alpha) as T - alpha T, the forward's expression
                        T2[h] = fma2(w, m1, T2[h]);
                    }
#pragma unroll
                    for (int i = 0; i < 9; ++i) v[i] = acc[i].x + acc[i].y;
                } else {
                    const Power<false> power(q, dx);
                    const float lim = s_floor[j];
#pragma unroll
                    for (int p = 0; p < kPixPerThread; ++p) {
                        const float dy = mu.y - fy[p];
                        const float pw = power.at(dy);
                        const bool act = idx < limit[p] && !(pw > 0.0f) && !(pw < lim);
                        const float raw = gaussian_weight<false>(q.w, pw);
                        const bool take = act && !(raw < kAlphaMin);
                        const float alpha = take ? fminf(kAlphaMax, raw) : 0.0f;
                        const float r = alpha < kAlphaMax ? alpha : 0.0f;
                        const float w = alpha * T[p];
                        const float inv = one_over<false>(1.0f - alpha);
                        const float G = gI[p][0] * cc[0] + gI[p][1] * cc[1] + gI[p][2] * cc[2];
                        const float dalpha = (P[p] + T[p] * G - S[p]) * inv;
#pragma unroll
                        for (int c = 0; c < 3; ++c) v[6 + c] += w * gI[p][c];
                        const float common = dalpha * r;
                        const float qx = fmaf(q.y, dy, qxdx);
                        const float qy = fmaf(q.z, dy, qydx);
                        const float cqx = common * qx, cqy = common * qy;
                        v[0] -= cqx;
                        v[1] -= cqy;
                        v[2] += cqx * qx;
                        v[3] += cqx * qy;
                        v[4] += cqy * qy;
                        v[5] += common;
                        v[9] += fabsf(cqx);
                        v[10] += fabsf(cqy);
                        P[p] += w * G;
                        T[p] = take ? T[p] * (1.0f - alpha) : T[p];
                    }
                }
                // d(cov a) and d(cov c) carry the factor 1/2 of the power, the
                // opacity logit the sigmoid's derivative o (1 - o) / o (exact)
                v[2] *= 0.5f;
                v[4] *= 0.5f;
                v[5] *= 1.0f - q.w;
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
        if ((reinterpret_cast<uintptr_t>(a.grad_out) & 15) == 0) {
            // one 16-byte vector reduction per group of four values (a Gaussian's 12
            // floats are a 48-byte row of the 16-byte aligned grad_out)
            for (int k = t; k < batch * (kVals / 4); k += kRasterThreads) {
                const float4 val = reinterpret_cast<const float4*>(s_acc)[k];
                if (val.x != 0.0f || val.y != 0.0f || val.z != 0.0f || val.w != 0.0f)
                    red_add_v4(a.grad_out + static_cast<int64_t>(s_id[k / (kVals / 4)]) * kVals + 4 * (k % (kVals / 4)),
                               val);
            }
        } else {
            for (int k = t; k < batch * kVals; k += kRasterThreads) {
                float val = s_acc[k];
                if (val != 0.0f) atomicAdd(a.grad_out + static_cast<int64_t>(s_id[k / kVals]) * kVals + k % kVals, val);
            }
        }
        __syncthreads();
    }
}

// The fast form with the forward's take flags: one warp per tile, eight pixels
// per lane (column px, rows y0 + 2p for p = 0..7, y0 = the tile's first or
// second row), evaluated as four packed pairs. A record some pixel of the tile
// took costs the tile one visit - one staging read, one set of column terms and
// one butterfly reduction - where a warp per 16x8 strip pays them twice for a
// record both strips took; and the reduced values go to their shared-memory
// slot with plain stores, since this warp alone writes them.
constexpr int kTilePix = 8;     // pixels per lane
constexpr int kTileBatch = 64;  // records staged per batch (two per lane)
constexpr int kTileChunks = kTileBatch / 32;

__global__ void __launch_bounds__(32) raster_backward_tile_kernel(RasterBackwardArgs a) {
    pdl_begin();
    __shared__ uint32_t s_id[kTileBatch];
    __shared__ float2 s_mean[kTileBatch];
    __shared__ float4 s_conic[kTileBatch];
    __shared__ float4 s_fast[kTileBatch];
    __shared__ float3 s_color[kTileBatch];
    __shared__ __align__(16) float s_acc[kTileBatch * kVals];

    const int lane = threadIdx.x;
    const int tile = blockIdx.x;
    const int tx = tile % a.cam.tile_count_x, ty = tile / a.cam.tile_count_x;
    const int px = tx * kTile + (lane & 15);
    const int y0 = ty * kTile + (lane >> 4);
    const float fx = static_cast<float>(px);
    const int64_t begin = a.tile_offsets[tile];
    const int64_t end_all = a.tile_offsets[tile + 1];

    // per pixel pair (2h, 2h + 1): -y, T, P - S (P = dL/dcolour . colour in
    // front of the record, S = dL/dcolour . final colour) and dL/dcolour
    float2 nfy2[kTilePix / 2], T2[kTilePix / 2], P2[kTilePix / 2], gI2[kTilePix / 2][3];
    int limit[kTilePix];
    int my_bound = 0;
#pragma unroll
    for (int p = 0; p < kTilePix; ++p) {
        const int py = y0 + 2 * p;
        float gi[3] = {0.0f, 0.0f, 0.0f};
        float S = 0.0f;
        limit[p] = 0;
        if (px < a.cam.width && py < a.cam.height) {
            const int64_t pix = static_cast<int64_t>(py) * a.cam.width + px;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                gi[c] = a.image_grad[pix * 3 + c];
                S += gi[c] * a.image[pix * 3 + c];
            }
            limit[p] = a.contributors[pix];
        }
        my_bound = max(my_bound, limit[p]);
        const int h = p >> 1;
        if (p & 1) {
            nfy2[h].y = -static_cast<float>(py);
            P2[h].y = -S;
#pragma unroll
            for (int c = 0; c < 3; ++c) gI2[h][c].y = gi[c];
        } else {
            nfy2[h].x = -static_cast<float>(py);
            P2[h].x = -S;
#pragma unroll
            for (int c = 0; c < 3; ++c) gI2[h][c].x = gi[c];
        }
        T2[h] = pk(1.0f);
    }
    // the replay ends at the tile's largest bound
    const int bound = __reduce_max_sync(0xffffffffu, my_bound);
    const int64_t end = begin + min(static_cast<int64_t>(bound), end_all - begin);
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
    const int low = (b2 ? 2 : 0) + (b1 ? 1 : 0);
    const int field = (b4 ? 6 : 0) + (b3 ? 3 : 0) + low;
    const bool writer = (lane & 1) == 0 && low < 3 && field < 11;

    for (int64_t base = begin; base < end; base += kTileBatch) {
        const int batch = static_cast<int>(min(static_cast<int64_t>(kTileBatch), end - base));
        // stage two records per lane; the take flags of the batch (a record some
        // pixel of the tile took in the forward pass) become two ballots
        uint32_t took[kTileChunks];
#pragma unroll
        for (int h = 0; h < kTileChunks; ++h) {
            const int slot = lane + h * 32;
            bool flag = false;
            if (slot < batch) {
                const uint32_t id = __ldg(a.tile_ids + base + slot);
                s_id[slot] = id;
                const float2 mean = __ldg(a.means + id);
                const float4 q = __ldg(a.conic_opacity + id);
                s_mean[slot] = mean;
                s_conic[slot] = q;
                const float* c = reinterpret_cast<const float*>(a.colors) + 3ull * id;
                s_color[slot] = make_float3(__ldg(c), __ldg(c + 1), __ldg(c + 2));
                s_fast[slot] = fast_record(q);
                const int64_t r = base + slot;
                const uint32_t bit = 1u << (r & 31);
                flag = ((a.record_warps[r >> 5] | a.record_warps[a.record_words + (r >> 5)]) & bit) != 0;
            }
            took[h] = __ballot_sync(0xffffffffu, flag);
        }
        for (int k = lane; k < kTileBatch * kVals; k += 32) s_acc[k] = 0.0f;
        __syncwarp();
        const int rel = static_cast<int>(base - begin);
        const int wend = min(batch, bound - rel);  // records below the tile's bound
#pragma unroll 1
        for (int h = 0; h < kTileChunks; ++h) {
            const int lim = wend - h * 32;
            if (lim <= 0) break;
            uint32_t m = lim < 32 ? took[h] & ((1u << lim) - 1u) : took[h];
            while (m) {
                const int j = h * 32 + __ffs(m) - 1;
                m &= m - 1;
                const int idx = rel + j;
                const float2 mu = s_mean[j];
                const float4 q = s_conic[j];
                const float3 col = s_color[j];
                const float4 kf = s_fast[j];
                const float dx = mu.x - fx;
                const float qxdx = q.x * dx, qydx = q.y * dx;
                const float Ax = fmaf(kf.x * dx, dx, kf.w), Bx = kf.y * dx;
                const float2 m1 = pk(-1.0f), one = pk(1.0f);
                float2 acc[9];
#pragma unroll
                for (int i = 0; i < 9; ++i) acc[i] = pk(0.0f);
                float abs_u = 0.0f, abs_v = 0.0f;
#pragma unroll
                for (int hp = 0; hp < kTilePix / 2; ++hp) {
                    const float2 dy = add2(pk(mu.y), nfy2[hp]);
                    const float2 pw2 = fma2(fma2(pk(kf.z), dy, pk(Bx)), dy, pk(Ax));
                    const bool take0 = idx < limit[2 * hp] && pw2.x >= kLog2AlphaMin;
                    const bool take1 = idx < limit[2 * hp + 1] && pw2.y >= kLog2AlphaMin;
                    float2 alpha;
                    alpha.x = take0 ? fminf(kAlphaMax, ex2_approx(pw2.x)) : 0.0f;
                    alpha.y = take1 ? fminf(kAlphaMax, ex2_approx(pw2.y)) : 0.0f;
                    // d alpha / d power: raw below the clamp, 0 when clamped or not taken
                    const float2 r = make_float2(alpha.x < kAlphaMax ? alpha.x : 0.0f,
                                                 alpha.y < kAlphaMax ? alpha.y : 0.0f);
                    const float2 w = mul2(alpha, T2[hp]);
                    const float2 om = fma2(alpha, m1, one);  // 1 - alpha
                    const float2 inv = make_float2(one_over<true>(om.x), one_over<true>(om.y));
                    float2 G = mul2(gI2[hp][0], pk(col.x));
                    G = fma2(gI2[hp][1], pk(col.y), G);
                    G = fma2(gI2[hp][2], pk(col.z), G);
                    // dL/dalpha = (dL/dC . (colour in front + T c - final)) / (1 - alpha)
                    const float2 dalpha = mul2(fma2(T2[hp], G, P2[hp]), inv);
#pragma unroll
                    for (int c = 0; c < 3; ++c) acc[6 + c] = fma2(w, gI2[hp][c], acc[6 + c]);
                    const float2 common = mul2(dalpha, r);
                    const float2 qx = fma2(pk(q.y), dy, pk(qxdx));
                    const float2 qy = fma2(pk(q.z), dy, pk(qydx));
                    const float2 cqx = mul2(common, qx), cqy = mul2(common, qy);
                    acc[0] = fma2(cqx, m1, acc[0]);
                    acc[1] = fma2(cqy, m1, acc[1]);
                    acc[2] = fma2(cqx, qx, acc[2]);  // halved once per record below
                    acc[3] = fma2(cqx, qy, acc[3]);
                    acc[4] = fma2(cqy, qy, acc[4]);  // halved once per record below
                    acc[5] = add2(acc[5], common);   // times (1 - o) once per record below
                    abs_u += fabsf(cqx.x) + fabsf(cqx.y);
                    abs_v += fabsf(cqy.x) + fabsf(cqy.y);
                    P2[hp] = fma2(w, G, P2[hp]);
                    T2[hp] = fma2(w, m1, T2[hp]);  // T - alpha T, the fast forward's expression
                }
                float v[kVals];
#pragma unroll
                for (int i = 0; i < 9; ++i) v[i] = acc[i].x + acc[i].y;
                v[9] = abs_u;
                v[10] = abs_v;
                v[11] = 0.0f;
                v[2] *= 0.5f;
                v[4] *= 0.5f;
                v[5] *= 1.0f - q.w;
                // butterfly reduce-scatter of the 12 slots (slot 11 is padding)
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
                // one lane per value; no other warp writes this batch's slots
                if (writer && k1 != 0.0f) s_acc[j * kVals + field] = k1;
            }
        }
        __syncwarp();
        if ((reinterpret_cast<uintptr_t>(a.grad_out) & 15) == 0) {
            for (int k = lane; k < batch * (kVals / 4); k += 32) {
                const float4 val = reinterpret_cast<const float4*>(s_acc)[k];
                if (val.x != 0.0f || val.y != 0.0f || val.z != 0.0f || val.w != 0.0f)
                    red_add_v4(a.grad_out + static_cast<int64_t>(s_id[k / (kVals / 4)]) * kVals + 4 * (k % (kVals / 4)),
                               val);
            }
        } else {
            for (int k = lane; k < batch * kVals; k += 32) {
                const float val = s_acc[k];
                if (val != 0.0f) atomicAdd(a.grad_out + static_cast<int64_t>(s_id[k / kVals]) * kVals + k % kVals, val);
            }
        }
        __syncwarp();
    }
}

}  // namespace

int launch_raster_backward(const RasterBackwardArgs& a, cudaStream_t stream) {
    int64_t tiles = static_cast<int64_t>(a.cam.tile_count_x) * a.cam.tile_count_y;
    if (tiles <= 0) return GSN_OK;
    if (!a.contributors) return GSN_ERR_INVALID_ARGUMENT;
    const unsigned grid = static_cast<unsigned>(tiles);
    if (a.fast && a.record_warps) launch_step(raster_backward_tile_kernel, grid, 32, 0, stream, a);
    else if (a.fast) launch_step(raster_backward_kernel<true>, grid, kRasterThreads, 0, stream, a);
    else launch_step(raster_backward_kernel<false>, grid, kRasterThreads, 0, stream, a);
    return launched(1);
}

}  // namespace gsn
