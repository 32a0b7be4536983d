// (f) Per-Gaussian update: view-space statistics, chain rule from the
// screen-space gradients to the 58 parameters, and Adam - fused into one pass
// over the SoA parameter block.
//
// The reference runs these as four launches around a 58 x N gradient buffer
// that is zeroed, written in place and read back (solver.cu:468-689, 862-923).
// Here one thread owns one Gaussian: it reads its 12 screen-space values, keeps
// the 58 parameter gradients in registers (the SH ones are formed on the fly as
// dL/dcolour * basis) and streams p, m, v once. That removes the 58 x N gradient
// round trip (3 x 232 B per Gaussian) from the largest HBM consumer of the step.
//
// The chain-rule arithmetic mirrors MapGaussianGradientsKernel (solver.cu:492-623)
// expression for expression, so for identical screen-space input the mapped
// gradients are bit-identical to the reference's; Adam follows
// UpdateGaussiansKernel (solver.cu:651-689).
#include "common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

struct Chain {
    float g[10];      // position 0-2, log-scale 3-5, axis-angle 6-8, opacity 9
    float basis[16];  // SH basis at the view direction
    float grgb[3];    // dL/dcolour, zero where the unclamped colour is negative
};

template <int D, bool kBf16>
__device__ __forceinline__ void sh_with_derivatives(const float* __restrict__ p, int64_t N, int i, const gsn_camera& cam,
                                                    float* basis, float* color, float* dcol) {
    constexpr int s = (D + 1) * (D + 1);
    float dir[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        dir[a] = p[a * N + i];
#pragma unroll
        for (int b = 0; b < 3; ++b) dir[a] += cam.R_c_w[b * 3 + a] * cam.t_c_w[b];
    }
    float il = rsqrtf(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    float x = dir[0] * il, y = dir[1] * il, z = dir[2] * il;
    float der[s * 3];
#pragma unroll
    for (int k = 0; k < s * 3; ++k) der[k] = 0.0f;
    basis[0] = kSh0;
    if (D >= 1) {
        basis[1] = -kSh1 * y;
        basis[2] = kSh1 * z;
        basis[3] = -kSh1 * x;
        der[4] = -kSh1;
        der[8] = kSh1;
        der[9] = -kSh1;
    }
    if (D >= 2) {
        constexpr float c = kSh2a, d = kSh2b, e = kSh2c;
        basis[4] = c * x * y;
        basis[5] = -c * y * z;
        basis[6] = d * (2 * z * z - x * x - y * y);
        basis[7] = -c * x * z;
        basis[8] = e * (x * x - y * y);
        der[12] = c * y;
        der[13] = c * x;
        der[16] = -c * z;
        der[17] = -c * y;
        der[18] = -2 * d * x;
        der[19] = -2 * d * y;
        der[20] = 4 * d * z;
        der[21] = -c * z;
        der[23] = -c * x;
        der[24] = 2 * e * x;
        der[25] = -2 * e * y;
    }
    if (D >= 3) {
        constexpr float a = -kSh3a, b = kSh3b, c = -kSh3c, d = kSh3d, e = kSh3e;
        basis[9] = a * y * (3 * x * x - y * y);
        basis[10] = b * x * y * z;
        basis[11] = c * y * (4 * z * z - x * x - y * y);
        basis[12] = d * z * (2 * z * z - 3 * x * x - 3 * y * y);
        basis[13] = c * x * (4 * z * z - x * x - y * y);
        basis[14] = e * z * (x * x - y * y);
        basis[15] = a * x * (x * x - 3 * y * y);
        der[27] = 6 * a * x * y;
        der[28] = 3 * a * (x * x - y * y);
        der[30] = b * y * z;
        der[31] = b * x * z;
        der[32] = b * x * y;
        der[33] = -2 * c * x * y;
        der[34] = c * (4 * z * z - x * x - 3 * y * y);
        der[35] = 8 * c * y * z;
        der[36] = -6 * d * x * z;
        der[37] = -6 * d * y * z;
        der[38] = d * (6 * z * z - 3 * x * x - 3 * y * y);
        der[39] = c * (4 * z * z - 3 * x * x - y * y);
        der[40] = -2 * c * x * y;
        der[41] = 8 * c * x * z;
        der[42] = 2 * e * x * z;
        der[43] = -2 * e * y * z;
        der[44] = e * (x * x - y * y);
        der[45] = 3 * a * (x * x - y * y);
        der[46] = -6 * a * x * y;
    }
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float value = 0.0f;
        float dv[3] = {0.0f, 0.0f, 0.0f};
        float coefs[s];
        load_sh_coefs<kBf16, s>(p, N, ch * kShStride, i, coefs);
#pragma unroll
        for (int j = 0; j < s; ++j) {
            const float coef = coefs[j];
            value += coef * basis[j];
#pragma unroll
            for (int a2 = 0; a2 < 3; ++a2) dv[a2] += coef * der[j * 3 + a2];
        }
        color[ch] = value + 0.5f;
        float radial = dv[0] * x + dv[1] * y + dv[2] * z;
        dcol[ch * 3] = (dv[0] - radial * x) * il;
        dcol[ch * 3 + 1] = (dv[1] - radial * y) * il;
        dcol[ch * 3 + 2] = (dv[2] - radial * z) * il;
    }
}

// Chain rule of solver.cu:512-622 for one Gaussian with screen gradients in[0..8].
template <int D, bool kBf16>
__device__ __forceinline__ void chain_rule(const float* __restrict__ p, int64_t N, int i, const gsn_camera& cam,
                                           const float in[9], Chain& out) {
    float rot[9], crot[9], cov[9], pos[3], s2[3];
    axis_angle_to_matrix(p[(GSN_ROTATION_INDEX + 0) * N + i], p[(GSN_ROTATION_INDEX + 1) * N + i],
                         p[(GSN_ROTATION_INDEX + 2) * N + i], rot);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        pos[r] = cam.t_c_w[r];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            pos[r] += cam.R_c_w[r * 3 + c] * p[static_cast<int64_t>(c) * N + i];
            crot[r * 3 + c] = cam.R_c_w[r * 3] * rot[c] + cam.R_c_w[r * 3 + 1] * rot[3 + c] +
                              cam.R_c_w[r * 3 + 2] * rot[6 + c];
        }
        float sc = expf(p[static_cast<int64_t>(GSN_LOG_SCALE_INDEX + r) * N + i]);
        s2[r] = sc * sc;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cov[r * 3 + c] = 0;
#pragma unroll
            for (int j = 0; j < 3; ++j) cov[r * 3 + c] += crot[r * 3 + j] * s2[j] * crot[c * 3 + j];
        }
    float iz = 1.0f / pos[2];
    float nx = pos[0] * iz, ny = pos[1] * iz;
    float lx = 1.3f * 0.5f * cam.width / cam.fx;
    float ly = 1.3f * 0.5f * cam.height / cam.fy;
    float jx = fminf(fmaxf(nx, -lx), lx);
    float jy = fminf(fmaxf(ny, -ly), ly);
    float P[6] = {cam.fx * iz, 0, -cam.fx * jx * iz, 0, cam.fy * iz, -cam.fy * jy * iz};
    float PV[6] = {}, LP[6] = {};
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                PV[r * 3 + c] += P[r * 3 + j] * cov[j * 3 + c];
                LP[r * 3 + c] += P[r * 3 + j] * crot[j * 3 + c];
            }
    float color[3], dcol[9];
    sh_with_derivatives<D, kBf16>(p, N, i, cam, out.basis, color, dcol);
    float right[3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        float dx = cam.R_c_w[axis], dy = cam.R_c_w[3 + axis], dz = cam.R_c_w[6 + axis];
        float du = (dx - nx * dz) * iz;
        float dv = (dy - ny * dz) * iz;
        float djx = nx >= -lx && nx <= lx ? du : 0;
        float djy = ny >= -ly && ny <= ly ? dv : 0;
        float delta[6] = {-cam.fx * dz * iz * iz, 0, -cam.fx * (djx - jx * dz * iz) * iz,
                          0, -cam.fy * dz * iz * iz, -cam.fy * (djy - jy * dz * iz) * iz};
        float daa = 0, dab = 0, ddd = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            daa += 2 * delta[j] * PV[j];
            dab += delta[j] * PV[3 + j] + delta[3 + j] * PV[j];
            ddd += 2 * delta[3 + j] * PV[3 + j];
        }
        float cg = in[0] * cam.fx * du + in[1] * cam.fy * dv + in[2] * daa + in[3] * dab + in[4] * ddd;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (color[c] >= 0) cg += in[6 + c] * dcol[c * 3 + axis];
        out.g[axis] = cg;
        float la = LP[axis], lb = LP[3 + axis];
        out.g[3 + axis] = 2 * s2[axis] * (in[2] * la * la + in[3] * la * lb + in[4] * lb * lb);
        int j = (axis + 1) % 3, k = (axis + 2) % 3;
        float diff = s2[j] - s2[k];
        right[axis] = diff * (2 * in[2] * LP[j] * LP[k] + in[3] * (LP[j] * LP[3 + k] + LP[k] * LP[3 + j]) +
                              2 * in[4] * LP[3 + j] * LP[3 + k]);
    }
    float w[3];
    float th2 = 0;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        w[axis] = p[static_cast<int64_t>(GSN_ROTATION_INDEX + axis) * N + i];
        th2 += w[axis] * w[axis];
    }
    float ca = 0.5f, cb = 1.0f / 6.0f;
    if (th2 > 1e-4f) {
        float th = sqrtf(th2);
        float hs = sinf(0.5f * th) / (0.5f * th);
        ca = 0.5f * hs * hs;
        cb = (th - sinf(th)) / (th2 * th);
    } else {
        ca -= th2 / 24.0f;
        cb -= th2 / 120.0f;
    }
    float cr[3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        int j = (axis + 1) % 3, k = (axis + 2) % 3;
        cr[axis] = w[j] * right[k] - w[k] * right[j];
    }
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        int j = (axis + 1) % 3, k = (axis + 2) % 3;
        out.g[6 + axis] = right[axis] + ca * cr[axis] + cb * (w[j] * cr[k] - w[k] * cr[j]);
    }
    out.g[9] = in[5];
#pragma unroll
    for (int c = 0; c < 3; ++c) out.grgb[c] = color[c] >= 0 ? in[6 + c] : 0.0f;
}

// Adam (UpdateGaussiansKernel arithmetic) on CNT consecutive rows starting at
// row0. All loads of the group are issued before any store, so the three
// streams of every row are in flight together; the parameter block and the
// two moment arrays never alias.
//
// The step lr * m_hat / (sqrt(v_hat) + 1e-15) uses the hardware approximate
// square root and divide (div.approx: 2 ulp for divisors in [2^-126, 2^126];
// the divisor here is >= 1e-15) instead of the IEEE-rounded sequences, whose
// special-case branches made this kernel branch-resolution bound (0.52 ms ->
// 0.40 ms at 1.2M Gaussians). Moments are formed exactly as in the reference;
// the parameter step differs from the reference's by at most a few ulps of
// the step.
// PTX sqrt.approx.f32 (relative error within 2^-23 on normal inputs).
__device__ __forceinline__ void prefetch_l2(const float* address) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(address));
}

__device__ __forceinline__ float sqrt_approx(float x) {
    float y;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// kLazy: the stored moments are first scaled by d1 = b1^k and d2 = b2^k, the
// decay of the k steps the Gaussian skipped under the visibility-masked update.
template <int CNT, bool kLazy = false>
__device__ __forceinline__ void adam_rows(float* __restrict__ P, float* __restrict__ M, float* __restrict__ V,
                                          int64_t N, int i, int row0, const float* g, const float* lr, float c1,
                                          float c2, float d1 = 1.0f, float d2 = 1.0f) {
    float p[CNT], m[CNT], v[CNT];
#pragma unroll
    for (int r = 0; r < CNT; ++r) {
        const int64_t idx = static_cast<int64_t>(row0 + r) * N + i;
        p[r] = P[idx];
        m[r] = M[idx];
        v[r] = V[idx];
        if constexpr (kLazy) {
            m[r] *= d1;
            v[r] *= d2;
        }
    }
#pragma unroll
    for (int r = 0; r < CNT; ++r) {
        float first = 0.9f * m[r] + 0.1f * g[r];
        float second = 0.999f * v[r] + 0.001f * g[r] * g[r];
        m[r] = first;
        v[r] = second;
        p[r] -= __fdividef(lr[r] * (first * c1), sqrt_approx(second * c2) + 1e-15f);
    }
#pragma unroll
    for (int r = 0; r < CNT; ++r) {
        const int64_t idx = static_cast<int64_t>(row0 + r) * N + i;
        P[idx] = p[r];
        M[idx] = m[r];
        V[idx] = v[r];
    }
}

// Precision form: the same step on bf16 SH pair rows (two coefficients of a
// Gaussian per 32-bit word, the parameters and both moments), computed in fp32
// and written back with stochastic rounding; coefficient by coefficient the
// noise stream is the one a row-by-row pass draws.
template <int PAIRS, bool kLazy = false>
__device__ __forceinline__ void adam_pairs_bf16(uint32_t* __restrict__ P, uint32_t* __restrict__ M,
                                                uint32_t* __restrict__ V, int64_t N, int i, int pair0,
                                                const float* g, const float* lr, float c1, float c2, uint32_t& rng,
                                                float d1 = 1.0f, float d2 = 1.0f) {
    // all of the group's words first (three per pair), so they are in flight
    // together; then pair by pair: widen, step, round, narrow, store
    uint32_t pw[PAIRS], mw[PAIRS], vw[PAIRS];
#pragma unroll
    for (int q = 0; q < PAIRS; ++q) {
        const int64_t idx = static_cast<int64_t>(pair0 + q) * N + i;
        pw[q] = P[idx];
        mw[q] = M[idx];
        vw[q] = V[idx];
    }
#pragma unroll
    for (int q = 0; q < PAIRS; ++q) {
        uint32_t bits[3] = {0u, 0u, 0u};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = 2 * q + h;
            float p = h ? bf16_hi(pw[q]) : bf16_lo(pw[q]);
            float m = h ? bf16_hi(mw[q]) : bf16_lo(mw[q]);
            float v = h ? bf16_hi(vw[q]) : bf16_lo(vw[q]);
            if constexpr (kLazy) {
                m *= d1;
                v *= d2;
            }
            const float first = 0.9f * m + 0.1f * g[r];
            const float second = 0.999f * v + 0.001f * g[r] * g[r];
            p -= __fdividef(lr[r] * (first * c1), sqrt_approx(second * c2) + 1e-15f);
            const uint32_t r1 = xorshift32(rng), r2 = xorshift32(rng);
            const int shift = 16 * h;
            bits[0] |= static_cast<uint32_t>(__bfloat16_as_ushort(bf16_stochastic(p, r1))) << shift;
            bits[1] |= static_cast<uint32_t>(__bfloat16_as_ushort(bf16_stochastic(first, r1 >> 16))) << shift;
            bits[2] |= static_cast<uint32_t>(__bfloat16_as_ushort(bf16_stochastic(second, r2))) << shift;
        }
        const int64_t idx = static_cast<int64_t>(pair0 + q) * N + i;
        P[idx] = bits[0];
        M[idx] = bits[1];
        V[idx] = bits[2];
    }
}

// log2 of Adam's decay rates, for the lazy decay b^k = 2^(k log2 b)
constexpr float kLog2Beta1 = -0.15200309344504995f;    // log2(0.9)
constexpr float kLog2Beta2 = -0.0014434168696687032f;  // log2(0.999)

template <int D, bool kBf16, bool kLazy>
__global__ void __launch_bounds__(256, 2) gaussian_update_kernel(GaussianUpdateArgs a) {
    pdl_begin();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t N = a.n;
    const float4* sg = reinterpret_cast<const float4*>(a.screen + static_cast<int64_t>(i) * 12);
    float4 s0 = sg[0], s1 = sg[1], s2 = sg[2];
    float in[9] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w, s2.x};
    float adu = s2.y, adv = s2.z;
    const bool visible = a.tile_counts[i] > 0;
    const gsn_camera cam = a.frame ? a.frame->cam : a.cam;
    // the moment rows Adam will read are fetched into L2 while the chain rule
    // computes: bytes in flight that cost no registers (the kernel runs at 128
    // registers and is bound by DRAM latency)
    if (a.m && !(a.sparse && !visible)) {
#pragma unroll 2
        for (int r = 0; r < physical_rows<kBf16>(); ++r) {
            prefetch_l2(a.m + static_cast<int64_t>(r) * N + i);
            prefetch_l2(a.v + static_cast<int64_t>(r) * N + i);
        }
    }

    // view-space statistics (solver.cu:468-490) and round accumulation
    // (density_controller.cu:280-295)
    float x = in[0] * (0.5f * cam.width);
    float y = in[1] * (0.5f * cam.height);
    float ax = adu * (0.5f * cam.width);
    float ay = adv * (0.5f * cam.height);
    float signed_len = sqrtf(x * x + y * y);
    float abs_len = sqrtf(ax * ax + ay * ay);
    if (a.stats) {
        a.stats[i] = signed_len;
        a.stats[N + i] = visible ? 1.0f : 0.0f;
    }
    if (a.abs_stats) {
        a.abs_stats[i] = abs_len;
        a.abs_stats[N + i] = adv;
    }
    if (a.grad_sums) {
        a.grad_sums[i] += signed_len;
        a.abs_sums[i] += abs_len;
        a.obs_counts[i] += visible ? 1u : 0u;
    }

    bool active = false;
#pragma unroll
    for (int k = 0; k < 9; ++k) active = active || in[k] != 0.0f;
    Chain ch;
    if (active) {
        chain_rule<D, kBf16>(a.params, N, i, cam, in, ch);
    } else {
#pragma unroll
        for (int k = 0; k < 10; ++k) ch.g[k] = 0.0f;
#pragma unroll
        for (int k = 0; k < 16; ++k) ch.basis[k] = 0.0f;
        ch.grgb[0] = ch.grgb[1] = ch.grgb[2] = 0.0f;
    }
    constexpr int K = (D + 1) * (D + 1);
    if (a.max_radius && visible) {
        // learned-policy statistics of the round (visible Gaussians only)
        const float depth = a.depths[i];
        a.max_radius[i] = fmaxf(a.max_radius[i], a.radii[i]);
        a.depth_sum[i] += depth;
        a.depth_sq[i] += depth * depth;
        float gm = 0.0f, gs = 0.0f, basis2 = 0.0f, rgb2 = 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            gm += ch.g[k] * ch.g[k];
            gs += ch.g[3 + k] * ch.g[3 + k];
            rgb2 += ch.grgb[k] * ch.grgb[k];
        }
#pragma unroll
        for (int k = 0; k < K; ++k) basis2 += ch.basis[k] * ch.basis[k];
        a.last_grad[i] = make_float4(sqrtf(gm), sqrtf(gs), fabsf(ch.g[9]), sqrtf(rgb2 * basis2));
    }
    if (a.grads_out) {
#pragma unroll
        for (int r = 0; r < 10; ++r) a.grads_out[r * N + i] = ch.g[r];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < kShStride; ++k)
                a.grads_out[(GSN_SH_INDEX + c * kShStride + k) * N + i] = k < K ? ch.grgb[c] * ch.basis[k] : 0.0f;
    }
    // visibility-masked (sparse) Adam: a Gaussian outside the view keeps its
    // parameters and moments (no momentum step, no moment decay; with lazy decay
    // the skipped steps' decay is applied at its next visible step, below)
    if (!a.m || (a.sparse && !visible)) return;
    float* __restrict__ P = a.params;
    float* __restrict__ M = a.m;
    float* __restrict__ V = a.v;
    const float lr0 = a.frame ? a.frame->position_lr : a.lr[0];
    const float c1 = a.frame ? a.frame->c1 : a.c1;
    const float c2 = a.frame ? a.frame->c2 : a.c2;
    const float lr_geo[10] = {lr0, lr0, lr0, a.lr[1], a.lr[1], a.lr[1], a.lr[2], a.lr[2], a.lr[2], a.lr[3]};
    // lazy moment decay: the moments decay as a dense step with a zero gradient
    // would have decayed them over the steps this Gaussian skipped (its
    // parameters do not take those steps' momentum moves); step 0 in last_step
    // means unknown (after a remap), which decays nothing
    float d1 = 1.0f, d2 = 1.0f;
    if constexpr (kLazy) {
        const uint32_t last = a.last_step[i];
        const uint32_t skipped = last != 0u && a.step > last + 1u ? a.step - last - 1u : 0u;
        d1 = exp2f(static_cast<float>(skipped) * kLog2Beta1);
        d2 = exp2f(static_cast<float>(skipped) * kLog2Beta2);
        a.last_step[i] = a.step;
    }
    adam_rows<10, kLazy>(P, M, V, N, i, 0, ch.g, lr_geo, c1, c2, d1, d2);
    if constexpr (kBf16) {
        // one group per colour channel: its 16 coefficients are 8 pair words
        // per array, the bytes in flight of the fp32 form's 8-row groups
        const uint32_t seed = a.frame ? a.frame->seed : a.seed;
        uint32_t rng = fmix32(static_cast<uint32_t>(i) * 0x9E3779B9u ^ fmix32(seed)) | 1u;
        float lr_sh[kShStride];
#pragma unroll
        for (int k = 0; k < kShStride; ++k) lr_sh[k] = k == 0 ? a.lr[4] : a.lr[5];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float g16[kShStride];
#pragma unroll
            for (int k = 0; k < kShStride; ++k) g16[k] = k < K ? ch.grgb[c] * ch.basis[k] : 0.0f;
            adam_pairs_bf16<kShStride / 2, kLazy>(reinterpret_cast<uint32_t*>(P), reinterpret_cast<uint32_t*>(M),
                                                  reinterpret_cast<uint32_t*>(V), N, i,
                                                  kGeometryRows + c * (kShStride / 2), g16, lr_sh, c1, c2, rng, d1,
                                                  d2);
        }
    } else {
        float lr_sh[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) lr_sh[k] = a.lr[5];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                float g8[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) g8[k] = half * 8 + k < K ? ch.grgb[c] * ch.basis[half * 8 + k] : 0.0f;
                lr_sh[0] = half == 0 ? a.lr[4] : a.lr[5];
                adam_rows<8, kLazy>(P, M, V, N, i, GSN_SH_INDEX + c * kShStride + half * 8, g8, lr_sh, c1, c2, d1,
                                    d2);
            }
        }
    }
}

// One 32-bit word per (physical row, Gaussian): an fp32 value, or a pair of
// bf16 SH moments in the precision layout (zero bits are two bf16 zeros).
__global__ void remap_moments_kernel(const int* __restrict__ parents, const float* __restrict__ prev_m,
                                     const float* __restrict__ prev_v, float* __restrict__ m, float* __restrict__ v,
                                     int prev_count, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int row = blockIdx.y;  // physical row
    const int parent = parents ? parents[i] : -1;
    const bool take = parent >= 0 && parent < prev_count;
    const int64_t dst = static_cast<int64_t>(row) * count + i;
    if (take) {
        const int64_t src = static_cast<int64_t>(row) * prev_count + parent;
        m[dst] = prev_m[src];
        v[dst] = prev_v[src];
    } else {
        m[dst] = 0.0f;
        v[dst] = 0.0f;
    }
}

template <bool kLazy>
int launch_update(const GaussianUpdateArgs& a, int d, dim3 grid, cudaStream_t stream) {
    if (a.bf16_sh) {
        switch (d) {
            case 0: launch_step(gaussian_update_kernel<0, true, kLazy>, grid, 256, 0, stream, a); break;
            case 1: launch_step(gaussian_update_kernel<1, true, kLazy>, grid, 256, 0, stream, a); break;
            case 2: launch_step(gaussian_update_kernel<2, true, kLazy>, grid, 256, 0, stream, a); break;
            default: launch_step(gaussian_update_kernel<3, true, kLazy>, grid, 256, 0, stream, a); break;
        }
    } else {
        switch (d) {
            case 0: launch_step(gaussian_update_kernel<0, false, kLazy>, grid, 256, 0, stream, a); break;
            case 1: launch_step(gaussian_update_kernel<1, false, kLazy>, grid, 256, 0, stream, a); break;
            case 2: launch_step(gaussian_update_kernel<2, false, kLazy>, grid, 256, 0, stream, a); break;
            default: launch_step(gaussian_update_kernel<3, false, kLazy>, grid, 256, 0, stream, a); break;
        }
    }
    return launched(1);
}

}  // namespace

int launch_gaussian_update(const GaussianUpdateArgs& a, int sh_degree, cudaStream_t stream) {
    if (a.n <= 0) return GSN_OK;
    dim3 grid(ceil_div(a.n, 256));
    const int d = sh_degree < 0 ? 0 : (sh_degree > 3 ? 3 : sh_degree);
    if (a.last_step && !a.sparse) return GSN_ERR_INVALID_ARGUMENT;  // lazy decay belongs to the sparse update
    if (a.last_step)
        return launch_update<true>(a, d, grid, stream);
    return launch_update<false>(a, d, grid, stream);
}

int launch_remap_moments(const int* parents, const float* prev_m, const float* prev_v, float* m, float* v,
                         int prev_count, int count, bool bf16_sh, cudaStream_t stream) {
    if (count <= 0) return GSN_OK;
    dim3 grid(ceil_div(count, 256), bf16_sh ? kPrecisionPhysicalRows : kParams);
    remap_moments_kernel<<<grid, 256, 0, stream>>>(parents, prev_m, prev_v, m, v, prev_count, count);
    return launched(1);
}

}  // namespace gsn
