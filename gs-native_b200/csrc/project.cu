// (a) Projection / preprocess: axis-angle -> rotation -> 3D covariance -> 2D conic,
// degree-3 SH colour and per-Gaussian tile-overlap counting.
//
// One thread per Gaussian over the 58 x N SoA parameter block, so every parameter
// row is read with fully coalesced 128-byte transactions. The arithmetic of the
// screen-space quantities (depth, u, v, radius and therefore the tile rectangle)
// follows the reference's expression order exactly (renderer.cu:108-221): tile
// keys, record counts and per-tile ranges must be bit-identical to the
// reference's own kernels.
#include "common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

// Evaluate the real SH basis of degree <= D at unit direction (x, y, z)
// (renderer.cu:68-106: same basis order and sign convention).
template <int D>
__device__ __forceinline__ void sh_basis(float x, float y, float z, float b[16]) {
    b[0] = kSh0;
    if (D < 1) return;
    b[1] = -kSh1 * y;
    b[2] = kSh1 * z;
    b[3] = -kSh1 * x;
    if (D < 2) return;
    float xx = x * x, yy = y * y, zz = z * z;
    float xy = x * y, yz = y * z, xz = x * z;
    b[4] = kSh2a * xy;
    b[5] = -kSh2a * yz;
    b[6] = kSh2b * (2.0f * zz - xx - yy);
    b[7] = -kSh2a * xz;
    b[8] = kSh2c * (xx - yy);
    if (D < 3) return;
    b[9] = -kSh3a * y * (3.0f * xx - yy);
    b[10] = kSh3b * xy * z;
    b[11] = -kSh3c * y * (4.0f * zz - xx - yy);
    b[12] = kSh3d * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    b[13] = -kSh3c * x * (4.0f * zz - xx - yy);
    b[14] = kSh3e * z * (xx - yy);
    b[15] = -kSh3a * x * (xx - 3.0f * yy);
}

// ---------------------------------------------------------------- exact tile culling
// A record (tile, Gaussian) can only change a pixel of its tile where
// alpha = o * exp(-q/2) >= 1/255, i.e. inside the ellipse q(d) <= 2 ln(255 o)
// (q(d) = A dx^2 + 2 B dx dy + C dy^2, conic (A, B, C), d = pixel - mean). The
// reference emits every tile of the 3-sigma rectangle; the culled form emits only
// the tiles whose pixel-centre rectangle meets that ellipse, widened as the blend
// kernels' alpha box is (2 % + 0.05 on Q plus a condition-number term, and a
// pixel pad), so a dropped record is one the per-pixel test rejects at every
// pixel of its tile: images, transmittance and gradients are unchanged.
//
// Per tile row the reachable columns form one interval: the ellipse's x-extent
// inside the band of the row's pixel centres, found at the band edge nearest to
// the ellipse's leftmost / rightmost point. Both functions are kept out of line
// so that the counting (projection) and the emitting kernel run one and the same
// instruction sequence on the same stored values and agree on every count.
struct CullShape {
    float mx, my;      // mean
    float B, inv_a;    // conic B, 1 / A
    float det, qa;     // A C - B^2, A * Q
    float hy, ys;      // y half-extent (padded), y of the rightmost point (negated)
    float pad_x;
    int mode;          // 0: reaches no pixel, 1: keep whole rows, 2: ellipse spans
};

__device__ __noinline__ CullShape cull_shape(float2 mean, float4 q) {
    CullShape s;
    s.mode = 0;
    s.mx = mean.x;
    s.my = mean.y;
    s.B = q.y;
    const float lo = 255.0f * q.w;
    if (!(lo > 1.0f)) return s;  // alpha can never reach 1/255
    s.mode = 1;
    const float det = q.x * q.z - q.y * q.y;
    const float tr = 0.5f * (q.x + q.z);
    const float disc = sqrtf(fmaxf(tr * tr - det, 0.0f));
    const float kappa = (tr + disc) / fmaxf(tr - disc, 1e-30f);
    if (!(det > 0.0f) || !(kappa < 1e5f) || !isfinite(mean.x) || !isfinite(mean.y) || !isfinite(lo)) return s;
    const float Q = 2.0f * __logf(lo) * (1.02f + 1e-6f * kappa) + 0.05f;
    const float hx = sqrtf(Q * q.z / det), hy = sqrtf(Q * q.x / det);
    if (!isfinite(hx) || !isfinite(hy)) return s;
    s.mode = 2;
    s.inv_a = 1.0f / q.x;
    s.det = det;
    s.qa = q.x * Q;
    s.hy = hy + 0.05f + 1e-3f * hy + 2e-5f * fabsf(mean.y);
    s.ys = q.y * hx / q.z;
    s.pad_x = 0.05f + 1e-3f * hx + 2e-5f * fabsf(mean.x);
    return s;
}

// Columns [x, y) of tile row ty (inside rect) that the record can reach.
__device__ __noinline__ int2 cull_row_span(CullShape s, int4 rect, int ty) {
    if (s.mode == 0) return make_int2(rect.x, rect.x);
    if (s.mode == 1) return make_int2(rect.x, rect.z);
    const float y0 = static_cast<float>(ty * kTile) - s.my, y1 = y0 + (kTile - 1);
    if (y0 > s.hy || y1 < -s.hy) return make_int2(rect.x, rect.x);
    const float yr = fminf(fmaxf(-s.ys, y0), y1), yl = fminf(fmaxf(s.ys, y0), y1);
    const float xr = (-s.B * yr + sqrtf(fmaxf(s.qa - s.det * yr * yr, 0.0f))) * s.inv_a;
    const float xl = (-s.B * yl - sqrtf(fmaxf(s.qa - s.det * yl * yl, 0.0f))) * s.inv_a;
    // tile tx holds pixel centres [16 tx, 16 tx + 15]
    const float c0 = floorf((s.mx + xl - s.pad_x) * (1.0f / kTile));
    const float c1 = floorf((s.mx + xr + s.pad_x) * (1.0f / kTile)) + 1.0f;
    const int a = static_cast<int>(fminf(fmaxf(c0, static_cast<float>(rect.x)), static_cast<float>(rect.z)));
    const int b = static_cast<int>(fminf(fmaxf(c1, static_cast<float>(rect.x)), static_cast<float>(rect.z)));
    return make_int2(a, max(a, b));
}

__device__ __forceinline__ int cull_count(float2 mean, float4 q, int4 rect) {
    const CullShape s = cull_shape(mean, q);
    if (s.mode == 0) return 0;
    if (s.mode == 1) return (rect.z - rect.x) * (rect.w - rect.y);
    int total = 0;
    for (int ty = rect.y; ty < rect.w; ++ty) {
        const int2 span = cull_row_span(s, rect, ty);
        total += span.y - span.x;
    }
    return total;
}

// Records of the culled counts in depth order. Four lanes serve a Gaussian and
// take its rows four at a time, one row each: a lane finds its row's column
// interval, the group's exclusive prefix of the interval widths (shuffles
// within the four lanes) places the row, and the four lanes write the group's
// records interleaved (consecutive lanes, consecutive slots).
// The loop runs the warp's largest number of row groups so every shuffle sees
// all 32 lanes.
__global__ void __launch_bounds__(256) emit_records_culled(const uint32_t* __restrict__ sorted_ids,
                                                           const int* __restrict__ record_start,
                                                           const int4* __restrict__ rects,
                                                           const float2* __restrict__ means,
                                                           const float4* __restrict__ conic_opacity, int n,
                                                           int tile_count_x, uint32_t* __restrict__ tile_keys,
                                                           uint32_t* __restrict__ record_ids, int64_t capacity,
                                                           int* overflow) {
    pdl_begin();
    const int64_t gidx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t p = gidx >> 2;
    const int sub = static_cast<int>(gidx & 3);
    bool active = p < n;
    int begin = 0, count = 0;
    uint32_t id = 0;
    if (active) {
        // the id is loaded with the offsets, ahead of the count checks
        begin = record_start[p];
        count = record_start[p + 1] - begin;
        id = sorted_ids[p];
        active = count > 0;
        // past the capacity the overflow flag is set and the records that still
        // fit are written (below), so every slot below min(total, capacity) -
        // all the sort and the blend read - holds a record
        if (active && begin + static_cast<int64_t>(count) > capacity) {
            if (sub == 0 && overflow) atomicExch(overflow, 1);
            active = begin < capacity;
        }
    }
    int4 r = make_int4(0, 0, 0, 0);
    CullShape s{};
    if (active) {
        r = rects[id];
        s = cull_shape(means[id], conic_opacity[id]);
    }
    const int groups = active ? (r.w - r.y + 3) / 4 : 0;
    const int rounds = __reduce_max_sync(0xffffffffu, groups);
    int k = 0;
    for (int g = 0; g < rounds; ++g) {
        const int ty = r.y + 4 * g + sub;
        int2 span = make_int2(0, 0);
        if (g < groups && ty < r.w) span = cull_row_span(s, r, ty);
        const int w = span.y - span.x;
        // exclusive prefix of the widths over the four lanes of this Gaussian
        int incl = w;
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o, 4);
            if (sub >= o) incl += y;
        }
        const int group_total = __shfl_sync(0xffffffffu, incl, 3, 4);
        // the group's four rows are one contiguous run of records; a record at
        // run position q of row i has tile q + base_i. The four lanes write the
        // run interleaved, so consecutive lanes write consecutive slots.
        const int base = ty * tile_count_x + span.x - (incl - w);
        const int e0 = __shfl_sync(0xffffffffu, incl, 0, 4), e1 = __shfl_sync(0xffffffffu, incl, 1, 4);
        const int e2 = __shfl_sync(0xffffffffu, incl, 2, 4);
        const int b0 = __shfl_sync(0xffffffffu, base, 0, 4), b1 = __shfl_sync(0xffffffffu, base, 1, 4);
        const int b2 = __shfl_sync(0xffffffffu, base, 2, 4), b3 = __shfl_sync(0xffffffffu, base, 3, 4);
        for (int q = sub; q < group_total && k + q < count && begin + k + q < capacity; q += 4) {
            const int row_base = q < e0 ? b0 : q < e1 ? b1 : q < e2 ? b2 : b3;
            tile_keys[begin + k + q] = static_cast<uint32_t>(row_base + q);
            record_ids[begin + k + q] = id;
        }
        k += group_total;
    }
    if (active && k != count && sub == 0 && overflow) atomicExch(overflow, 2);
}

// kBf16: precision form (bf16 SH rows; near-singular conics inverted in FP64).
// TW x TH: tile shape of the rectangle (16 x 16, the reference's, everywhere but
// the multi-view renderer's tile-shape sweep).
template <int D, bool kBf16, int TW = kTile, int TH = kTile>
__global__ void __launch_bounds__(256) project_kernel(const float* __restrict__ params,
                                                      gsn_camera cam_arg, const gsn_camera* __restrict__ cam_dev,
                                                      int n, ProjectOutputs out) {
    pdl_begin();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const gsn_camera cam = cam_dev ? *cam_dev : cam_arg;
    const int64_t N = n;
    out.tile_counts[i] = 0;
    if (out.cull_counts) out.cull_counts[i] = 0;
    out.depth_keys[i] = 0xFFFFFFFFu;
    if (out.radii) out.radii[i] = 0.0f;

    const float gx = __ldg(params + 0 * N + i);
    const float gy = __ldg(params + 1 * N + i);
    const float gz = __ldg(params + 2 * N + i);
    const float* R = cam.R_c_w;
    const float* t = cam.t_c_w;
    float px = R[0] * gx + R[1] * gy + R[2] * gz + t[0];
    float py = R[3] * gx + R[4] * gy + R[5] * gz + t[1];
    float z = R[6] * gx + R[7] * gy + R[8] * gz + t[2];
    float near = fmaxf(cam.near_depth, kNearFloor);
    if (z <= near || z > fmaxf(cam.far_depth, near)) return;

    float Rg[9];
    axis_angle_to_matrix(__ldg(params + 6 * N + i), __ldg(params + 7 * N + i),
                         __ldg(params + 8 * N + i), Rg);
    float s[3] = {expf(__ldg(params + 3 * N + i)), expf(__ldg(params + 4 * N + i)),
                  expf(__ldg(params + 5 * N + i))};
    // M = R_c_w * R_g * S, cov = M M^T.
    float M[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            M[r * 3 + c] = (R[r * 3] * Rg[c] + R[r * 3 + 1] * Rg[3 + c] + R[r * 3 + 2] * Rg[6 + c]) * s[c];
    float V[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            V[r * 3 + c] = M[r * 3] * M[c * 3] + M[r * 3 + 1] * M[c * 3 + 1] + M[r * 3 + 2] * M[c * 3 + 2];

    // Clamped perspective Jacobian.
    float lim_x = kFovClamp * 0.5f * cam.width / cam.fx;
    float lim_y = kFovClamp * 0.5f * cam.height / cam.fy;
    float cxz = fminf(fmaxf(px / z, -lim_x), lim_x) * z;
    float cyz = fminf(fmaxf(py / z, -lim_y), lim_y) * z;
    float J[6] = {cam.fx / z, 0.0f, -cam.fx * cxz / (z * z), 0.0f, cam.fy / z, -cam.fy * cyz / (z * z)};
    float JV[6];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            JV[r * 3 + c] = J[r * 3] * V[c] + J[r * 3 + 1] * V[3 + c] + J[r * 3 + 2] * V[6 + c];
    float a = JV[0] * J[0] + JV[1] * J[1] + JV[2] * J[2] + kLowPass;
    float b = JV[0] * J[3] + JV[1] * J[4] + JV[2] * J[5];
    float c = JV[3] * J[3] + JV[4] * J[4] + JV[5] * J[5] + kLowPass;
    float det = a * c - b * b;
    // precision form: when a*c and b^2 agree in their leading 12 bits the fp32
    // difference has lost them, so the determinant and the inverse are formed
    // in FP64 (the only FP64 use of the projection)
    bool singular64 = false;
    double det64 = 0.0;
    if constexpr (kBf16) {
        if (det < 2.44140625e-4f * (a * c)) {
            det64 = static_cast<double>(a) * c - static_cast<double>(b) * b;
            if (!(det64 > 0.0)) return;
            det = static_cast<float>(det64);
            singular64 = true;
        }
    }
    if (!(det > 0.0f) && !singular64) return;
    float mid = 0.5f * (a + c);
    float radius = ceilf(3.0f * sqrtf(mid + sqrtf(fmaxf(0.1f, mid * mid - det))));
    float u = cam.fx * px / z + cam.cx;
    float v = cam.fy * py / z + cam.cy;
    if (!isfinite(radius) || !isfinite(u) || !isfinite(v)) return;
    int4 rect;
    rect.x = static_cast<int>(fminf(cam.tile_count_x, fmaxf(0.0f, (u - radius) / TW)));
    rect.y = static_cast<int>(fminf(cam.tile_count_y, fmaxf(0.0f, (v - radius) / TH)));
    rect.z = static_cast<int>(fminf(cam.tile_count_x, fmaxf(0.0f, (u + radius + TW - 1) / TW)));
    rect.w = static_cast<int>(fminf(cam.tile_count_y, fmaxf(0.0f, (v + radius + TH - 1) / TH)));
    if (rect.x >= rect.z || rect.y >= rect.w) return;

    out.depths[i] = z;
    out.depth_keys[i] = __float_as_uint(z) >> out.depth_key_shift;  // z > 0: monotonic in z
    out.rects[i] = rect;
    out.tile_counts[i] = (rect.z - rect.x) * (rect.w - rect.y);
    if (out.radii) out.radii[i] = radius;
    float opacity = 1.0f / (1.0f + expf(-__ldg(params + 9 * N + i)));
    out.means[i] = make_float2(u, v);
    float4 conic;
    if (singular64) {
        const double inv64 = 1.0 / det64;
        conic = make_float4(static_cast<float>(c * inv64), static_cast<float>(-b * inv64),
                            static_cast<float>(a * inv64), opacity);
    } else {
        float det_inv = 1.0f / det;
        conic = make_float4(c * det_inv, -b * det_inv, a * det_inv, opacity);
    }
    out.conic_opacity[i] = conic;
    if constexpr (TW == kTile && TH == kTile) {
        if (out.cull_counts) out.cull_counts[i] = cull_count(make_float2(u, v), conic, rect);
    }

    // View direction from the camera centre, C = -R^T t.
    float dx = gx + R[0] * t[0] + R[3] * t[1] + R[6] * t[2];
    float dy = gy + R[1] * t[0] + R[4] * t[1] + R[7] * t[2];
    float dz = gz + R[2] * t[0] + R[5] * t[1] + R[8] * t[2];
    float inv_len = rsqrtf(dx * dx + dy * dy + dz * dz);
    float basis[16];
    sh_basis<D>(dx * inv_len, dy * inv_len, dz * inv_len, basis);
    constexpr int K = (D + 1) * (D + 1);
    float rgb[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float coef[K];
        load_sh_coefs<kBf16, K>(params, N, ch * kShStride, i, coef);
        float value = 0.0f;
#pragma unroll
        for (int k = 0; k < K; ++k) value += basis[k] * coef[k];
        rgb[ch] = fmaxf(value + 0.5f, 0.0f);
    }
    out.colors[i] = make_float3(rgb[0], rgb[1], rgb[2]);
}

template <bool kBf16>
void launch_project_layout(const float* params, int n, const gsn_camera& cam, const gsn_camera* cam_dev, int d,
                           const ProjectOutputs& out, cudaStream_t stream) {
    dim3 grid(ceil_div(n, 256));
    switch (d) {
        case 0: launch_step(project_kernel<0, kBf16>, grid, 256, 0, stream, params, cam, cam_dev, n, out); break;
        case 1: launch_step(project_kernel<1, kBf16>, grid, 256, 0, stream, params, cam, cam_dev, n, out); break;
        case 2: launch_step(project_kernel<2, kBf16>, grid, 256, 0, stream, params, cam, cam_dev, n, out); break;
        default: launch_step(project_kernel<3, kBf16>, grid, 256, 0, stream, params, cam, cam_dev, n, out); break;
    }
}

}  // namespace

template <int TW, int TH>
static void launch_project_tiles(const float* params, int n, const gsn_camera& cam, int d, const ProjectOutputs& out,
                          cudaStream_t stream) {
    dim3 grid(ceil_div(n, 256));
    switch (d) {
        case 0: launch_step(project_kernel<0, false, TW, TH>, grid, 256, 0, stream, params, cam, nullptr, n, out);
            break;
        case 1: launch_step(project_kernel<1, false, TW, TH>, grid, 256, 0, stream, params, cam, nullptr, n, out);
            break;
        case 2: launch_step(project_kernel<2, false, TW, TH>, grid, 256, 0, stream, params, cam, nullptr, n, out);
            break;
        default: launch_step(project_kernel<3, false, TW, TH>, grid, 256, 0, stream, params, cam, nullptr, n, out);
            break;
    }
}

int launch_project_tiled(const float* params, int n, const gsn_camera& cam, int tile_w, int tile_h, int sh_degree,
                         const ProjectOutputs& out, cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    const int d = sh_degree < 0 ? 0 : (sh_degree > 3 ? 3 : sh_degree);
    if (tile_w == 16 && tile_h == 16) launch_project_tiles<16, 16>(params, n, cam, d, out, stream);
    else if (tile_w == 16 && tile_h == 8) launch_project_tiles<16, 8>(params, n, cam, d, out, stream);
    else if (tile_w == 8 && tile_h == 8) launch_project_tiles<8, 8>(params, n, cam, d, out, stream);
    else return GSN_ERR_INVALID_ARGUMENT;
    return launched(1);
}

int launch_emit_records_culled(const uint32_t* sorted_ids, const int* record_start, const int4* rects,
                               const float2* means, const float4* conic_opacity, int n, int tile_count_x,
                               uint32_t* tile_keys, uint32_t* record_ids, int64_t capacity, int* overflow,
                               cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    launch_step(emit_records_culled, ceil_div(4ll * n, 256), 256, 0, stream, sorted_ids, record_start, rects, means,
                conic_opacity, n, tile_count_x, tile_keys, record_ids, capacity, overflow);
    return launched(1);
}

int launch_project(const float* params, int n, const gsn_camera& cam, const gsn_camera* cam_dev, int sh_degree,
                   bool bf16_sh, const ProjectOutputs& out, cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    const int d = sh_degree < 0 ? 0 : (sh_degree > 3 ? 3 : sh_degree);
    if (bf16_sh) launch_project_layout<true>(params, n, cam, cam_dev, d, out, stream);
    else launch_project_layout<false>(params, n, cam, cam_dev, d, out, stream);
    return launched(1);
}

}  // namespace gsn
