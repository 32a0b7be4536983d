// Shared pieces of the forward and backward tile kernels.
//
// Both kernels run one 64-thread CTA per 16x16 tile: thread t of warp w owns the
// four pixels (x, y0 + 2p), p = 0..3, with x = t % 16 and
// y0 = 8w + (t % 32) / 16, so warp w covers the 16x8 strip of rows 8w..8w+7.
// Records are staged in batches of 128 (two per thread).
#pragma once

#include "common.cuh"

namespace gsn {

constexpr int kRasterThreads = 64;
constexpr int kPixPerThread = 4;
constexpr int kRasterBatch = 128;

struct TileGeometry {
    int tile, tx, ty;
    int px;            // pixel column
    int py[kPixPerThread];
    float sx0, sx1, sy0, sy1;  // the warp's pixel strip
};

__device__ __forceinline__ TileGeometry tile_geometry(const gsn_camera& cam) {
    TileGeometry g;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    g.tile = blockIdx.x;
    g.tx = g.tile % cam.tile_count_x;
    g.ty = g.tile / cam.tile_count_x;
    g.px = g.tx * kTile + (lane & 15);
    const int y0 = g.ty * kTile + 8 * warp + (lane >> 4);
#pragma unroll
    for (int p = 0; p < kPixPerThread; ++p) g.py[p] = y0 + 2 * p;
    g.sx0 = static_cast<float>(g.tx * kTile);
    g.sx1 = g.sx0 + (kTile - 1);
    g.sy0 = static_cast<float>(g.ty * kTile + 8 * warp);
    g.sy1 = g.sy0 + 7.0f;
    return g;
}

// Conservative pixel-space box outside of which a record cannot reach
// alpha >= 1/255. With conic (A, B, C) and opacity o, alpha >= 1/255 needs
// q(d) = A dx^2 + 2 B dx dy + C dy^2 <= Q = 2 ln(255 o); the ellipse q <= Q has
// half-extents sqrt(Q * C / det) and sqrt(Q * A / det), det = AC - B^2.
// The bound is widened for the rounding of the per-pixel float evaluation, which
// can reach a few ulps of A dx^2 + C dy^2 (up to ~kappa * q for a conic with
// condition number kappa), so a culled record is one the exact per-pixel test
// would have skipped for every pixel of the box: culling never changes a result.
// A record that can never pass (255 o <= 1) gets an empty box; a degenerate or
// non-finite conic gets an unbounded one.
__device__ __forceinline__ float4 alpha_box(float2 mean, float4 q) {
    const float inf = __int_as_float(0x7f800000);
    float lo = 255.0f * q.w;
    if (!(lo > 1.0f)) return make_float4(inf, -inf, inf, -inf);
    float det = q.x * q.z - q.y * q.y;
    float tr = 0.5f * (q.x + q.z);
    float disc = sqrtf(fmaxf(tr * tr - det, 0.0f));
    float lmin = tr - disc, lmax = tr + disc;
    float kappa = lmax / fmaxf(lmin, 1e-30f);
    float Q = 2.0f * __logf(lo) * (1.02f + 1e-6f * kappa) + 0.05f;
    float hx = sqrtf(Q * q.z / det) * 1.001f + 0.05f;
    float hy = sqrtf(Q * q.x / det) * 1.001f + 0.05f;
    if (!(det > 0.0f) || !(kappa < 1e5f) || !isfinite(hx) || !isfinite(hy) || !isfinite(mean.x) ||
        !isfinite(mean.y))
        return make_float4(-inf, inf, -inf, inf);
    return make_float4(mean.x - hx, mean.x + hx, mean.y - hy, mean.y + hy);
}

// Power below which alpha = min(0.99, o * expf(power)) is certainly < 1/255:
// power < -ln(255 o) - 1e-3 gives o * e^power < e^-0.001 / 255, a relative gap
// far wider than the rounding of expf and of the product. -inf disables the test.
__device__ __forceinline__ float alpha_floor(float opacity) {
    float lo = 255.0f * opacity;
    if (!(lo > 0.0f) || !isfinite(lo)) return -__int_as_float(0x7f800000);
    return -logf(lo) - 1e-3f;
}

// Gaussian power -(A dx^2 + C dy^2) / 2 - B dx dy of a record at the pixels of
// one column (shared dx). The exact form evaluates the reference's expression
// per pixel (renderer.cu:300-303) so images match it bit for bit; the fast form
// (kFast) hoists the per-record terms and evaluates two FMAs per pixel, which
// moves the result by a few ulps - far inside the alpha floor's and the alpha
// box's margins, so every skip decision stays conservative.
template <bool kFast>
struct Power {
    float a, b, c;  // fast form: a + dy * (b + c * dy)
    float4 q;
    float dx;
    __device__ __forceinline__ Power(float4 conic, float delta_x) : q(conic), dx(delta_x) {
        if (kFast) {
            a = -0.5f * q.x * dx * dx;
            b = -q.y * dx;
            c = -0.5f * q.z;
        }
    }
    __device__ __forceinline__ float at(float dy) const {
        if (kFast) return fmaf(fmaf(c, dy, b), dy, a);
        return -0.5f * (q.x * dx * dx + q.z * dy * dy) - q.y * dx * dy;
    }
};

// o * e^power: the reference's expf in the exact form, the hardware exp2
// approximation (__expf) in the fast form.
template <bool kFast>
__device__ __forceinline__ float gaussian_weight(float opacity, float power) {
    return kFast ? opacity * __expf(power) : opacity * expf(power);
}

// 1 / x for x in [0.01, 1] (one minus a clamped alpha): the correctly rounded
// reciprocal in the exact form, the single hardware approximation (PTX
// rcp.approx, within an ulp) in the fast form.
template <bool kFast>
__device__ __forceinline__ float one_over(float x) {
    if (!kFast) return __frcp_rn(x);
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Fast-form record terms. The fast forms evaluate a record's alpha as
// ex2(pw2) with pw2 = log2(o) + log2(e) * power, the Gaussian power in log2
// units with the opacity folded in: per record k = (-log2(e) A / 2,
// -log2(e) B, -log2(e) C / 2, log2(o)), per (thread, record) the column terms
// Ax = k.x dx^2 + k.w and Bx = k.y dx, per pixel two FMAs
// pw2 = (k.z dy + Bx) dy + Ax and one MUFU ex2. A pixel takes the record when
// alpha >= 1/255, i.e. pw2 >= log2(1/255) (one compare; false for NaN; a
// record with o < 1/255 never passes since pw2 <= log2(o)). The reference's
// second test, power > 0, only catches rounding: projected conics are
// positive definite (the 2D covariance carries +0.3 on its diagonal and
// det <= 0 is culled), so the true power is never positive; the fast forms
// drop it, as evaluating it against log2(o) would reject pixels within an ulp
// of a Gaussian's centre. The forward and backward fast kernels share these
// expressions, so their take decisions agree.
constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLog2AlphaMin = -7.9943534368588578f;  // log2(1/255)

__device__ __forceinline__ float4 fast_record(float4 q) {
    return make_float4(-0.5f * kLog2e * q.x, -kLog2e * q.y, -0.5f * kLog2e * q.z, log2f(q.w));
}

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Packed FP32x2 arithmetic (sm_100: one instruction performs two IEEE
// round-to-nearest operations, each rounded as its scalar form). The fast forms
// evaluate a thread's four pixels as two pairs (pixels 2h and 2h + 1) with
// these, which halves the issue slots of their per-pixel arithmetic.
__device__ __forceinline__ float2 pk(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// Does the box of a record overlap the pixel rectangle [x0, x1] x [y0, y1]?
__device__ __forceinline__ bool box_hits(float4 b, float x0, float x1, float y0, float y1) {
    return b.x <= x1 && b.y >= x0 && b.z <= y1 && b.w >= y0;
}

}  // namespace gsn
