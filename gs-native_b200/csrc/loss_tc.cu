// (e) Precision form of the fused L1 + SSIM loss gradient: the separable 11x11
// Gaussian window runs as banded-Toeplitz GEMMs on the tcgen05 tensor cores.
//
// Same loss and gradient as loss.cu (L = 0.8 mean|I - T| + 0.2 (1 - mean SSIM),
// zero padding, C1 = 1e-4, C2 = 9e-4; dL/dI = (0.8 sign(I - T) - 0.2 (F(pa) +
// T F(pb) + 2 I F(pc))) / 3P with F the 2D window and pa, pb, pc the per-centre
// SSIM partials). Every filter pass is a matrix product with a banded Toeplitz
// matrix of the 11 window weights:
//   horizontal  H = X * Wh        (X: 128 rows x 64 columns, Wh: 64 x 64)
//   vertical    V = Wv * H        (Wv: 128 x 128)
// The operands are fp32 values split into bf16 hi + lo parts (x = hi + lo with
// |lo| <= 2^-9 |x|); each product is accumulated as hi*hi + hi*lo + lo*hi in
// fp32 tensor memory, which leaves a relative error of about 2^-16 per pass.
//
// Work item: one 108 x 44 block of output pixels of one colour channel. Its
// input block is 128 x 64 pixels (10-pixel halo); moments are valid on the
// inner 118 x 54 centres and the back-filtered partials on the 108 x 44 output
// pixels. CTAs are persistent (one per SM, 512 threads: four 16-column groups
// per block row) and keep the two Toeplitz operands (80 KB) resident in shared
// memory.
// Tensor memory: the five filtered moments (5 x 64 columns), one 64-column
// scratch for the horizontal pass and one for the vertical pass of a partial.
// The FP64 loss sums (sum |I - T|, sum SSIM, sum (I - T)^2) are reduced as in
// loss.cu.
#include <cuda_bf16.h>

#include <mutex>

#include "common.cuh"
#include "kernels.h"
#include "tcgen05.cuh"

namespace gsn {

namespace {

__constant__ float c_window_tc[11] = {1.028380120e-03f, 7.598758210e-03f, 3.600077330e-02f, 1.093606870e-01f,
                                      2.130055430e-01f, 2.660117150e-01f, 2.130055430e-01f, 1.093606870e-01f,
                                      3.600077330e-02f, 7.598758210e-03f, 1.028380120e-03f};

constexpr int kRows = 128;            // block rows (MMA M, tensor-memory lanes)
constexpr int kCols = 64;             // block columns (MMA N)
constexpr int kOutRows = kRows - 20;  // 108 output rows per block
constexpr int kOutCols = kCols - 20;  // 44 output columns per block
constexpr int kRawStride = kCols + 1; // padded fp32 row stride of the raw tiles
constexpr float kC1 = 0.0001f;
constexpr float kC2 = 0.0009f;
constexpr long long kWaitCycles = 2000000000LL;
constexpr int kGroups = 4;                       // column groups per block row
constexpr int kGroupCols = kCols / kGroups;      // 16 columns per thread
constexpr int kThreads = kRows * kGroups;        // 512 threads

// shared memory map (bytes)
constexpr uint32_t kWvBytes = kRows * kRows * 2;         // 32 KB per part
constexpr uint32_t kWhBytes = kCols * kCols * 2;         //  8 KB per part
constexpr uint32_t kABytes = kRows * kCols * 2;          // 16 KB per part: X (128 x 64, K = 64)
constexpr uint32_t kBBytes = kCols * kRows * 2;          // 16 KB per part: H^T (64 x 128, K = 128)
constexpr uint32_t kOffWvHi = 0;
constexpr uint32_t kOffWvLo = kOffWvHi + kWvBytes;
constexpr uint32_t kOffWhHi = kOffWvLo + kWvBytes;
constexpr uint32_t kOffWhLo = kOffWhHi + kWhBytes;
constexpr uint32_t kOffAHi = kOffWhLo + kWhBytes;
constexpr uint32_t kOffALo = kOffAHi + kABytes;
constexpr uint32_t kOffBHi = kOffALo + kABytes;
constexpr uint32_t kOffBLo = kOffBHi + kBBytes;
constexpr uint32_t kOffRawI = kOffBLo + kBBytes;
constexpr uint32_t kOffRawT = kOffRawI + kRows * kRawStride * 4;
constexpr uint32_t kSmemBytes = kOffRawT + kRows * kRawStride * 4;  // 214,016 B

// tensor-memory columns
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kColMoments = 0;    // 5 x 64
constexpr uint32_t kColH = 320;        // horizontal-pass result
constexpr uint32_t kColV = 384;        // vertical pass of a partial

__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 a, __nv_bfloat16 b) {
    return static_cast<uint32_t>(__bfloat16_as_ushort(a)) | (static_cast<uint32_t>(__bfloat16_as_ushort(b)) << 16);
}

// Writes 16 columns [c0, c0 + 16) of row r of a 128 x 64 A operand (K-major,
// K = 64) as hi and lo parts: two 16-byte stores per part.
__device__ __forceinline__ void store_a(uint8_t* smem, int r, int c0, const float* v) {
#pragma unroll
    for (int h8 = 0; h8 < 16; h8 += 8) {
        __nv_bfloat16 h[8], l[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) split_bf16(v[h8 + j], h[j], l[j]);
        const uint32_t off = tc::kmajor_offset(r, c0 + h8, kCols);
        *reinterpret_cast<uint4*>(smem + kOffAHi + off) =
            make_uint4(pack2(h[0], h[1]), pack2(h[2], h[3]), pack2(h[4], h[5]), pack2(h[6], h[7]));
        *reinterpret_cast<uint4*>(smem + kOffALo + off) =
            make_uint4(pack2(l[0], l[1]), pack2(l[2], l[3]), pack2(l[4], l[5]), pack2(l[6], l[7]));
    }
}

// Issues the horizontal pass H = X * Wh (M 128, N 64, K 64) into tensor memory.
__device__ __forceinline__ void issue_horizontal(const uint8_t* smem, uint32_t tmem_h) {
    const uint32_t idesc = tc::idesc_bf16_f32(kRows, kCols);
    const uint32_t base = tc::smem_u32(smem);
    constexpr uint32_t sbo = kCols * 16;  // K = 64
#pragma unroll 1
    for (int k = 0; k < kCols / 16; ++k) {
        const uint32_t o = k * 256;
        const uint64_t ahi = tc::smem_desc(base + kOffAHi + o, 128, sbo);
        const uint64_t alo = tc::smem_desc(base + kOffALo + o, 128, sbo);
        const uint64_t bhi = tc::smem_desc(base + kOffWhHi + o, 128, sbo);
        const uint64_t blo = tc::smem_desc(base + kOffWhLo + o, 128, sbo);
        tc::mma_bf16(tmem_h, ahi, bhi, idesc, k > 0);
        tc::mma_bf16(tmem_h, ahi, blo, idesc, true);
        tc::mma_bf16(tmem_h, alo, bhi, idesc, true);
    }
}

// Issues the vertical pass V = Wv * H (M 128, N 64, K 128) with H staged as
// an MN-major B operand (instruction-descriptor bit 16).
__device__ __forceinline__ void issue_vertical(const uint8_t* smem, uint32_t tmem_v) {
    const uint32_t idesc = tc::idesc_bf16_f32(kRows, kCols) | (1u << 16);
    const uint32_t base = tc::smem_u32(smem);
    constexpr uint32_t sbo = kRows * 16;  // K = 128
#pragma unroll 1
    for (int k = 0; k < kRows / 16; ++k) {
        const uint32_t o = k * 256;
        const uint64_t ahi = tc::smem_desc(base + kOffWvHi + o, 128, sbo);
        const uint64_t alo = tc::smem_desc(base + kOffWvLo + o, 128, sbo);
        // MN-major B: LBO = 128 bytes between K groups, SBO = 2048 between N groups
        const uint64_t bhi = tc::smem_desc(base + kOffBHi + o, 128, sbo);
        const uint64_t blo = tc::smem_desc(base + kOffBLo + o, 128, sbo);
        tc::mma_bf16(tmem_v, ahi, bhi, idesc, k > 0);
        tc::mma_bf16(tmem_v, ahi, blo, idesc, true);
        tc::mma_bf16(tmem_v, alo, bhi, idesc, true);
    }
}

struct Sync {
    uint64_t* bar;
    uint32_t phase;
    bool ok;
};

// All threads: make the staged operands visible to the tensor core and let
// thread 0 issue a pass (no completion wait).
template <class Issue>
__device__ __forceinline__ void issue(Sync& s, Issue body) {
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc::fence_after_sync();
        if (s.ok) body();
    }
}

// Thread 0 commits everything issued so far; all threads wait (bounded).
__device__ __forceinline__ void commit_wait(Sync& s) {
    if (threadIdx.x == 0) tc::commit(s.bar);
    const bool done = tc::mbar_wait(s.bar, s.phase, kWaitCycles);
    s.phase ^= 1u;
    s.ok = __syncthreads_and(done) && s.ok;
    tc::fence_after_sync();
}

// H (tensor memory) -> B operand of the vertical pass in the canonical
// MN-major layout (no swizzle): element (n = column c, k = row r) at
// (c / 8) * 2048 + (r / 8) * 128 + (r % 8) * 16 + (c % 8) * 2, i.e. 8 columns
// of one row are 16 contiguous bytes, so each thread stores its own row with
// 16-byte stores and no transpose (LBO = 128 between 8-row groups of K,
// SBO = 2048 between 8-column groups of N).
__device__ __forceinline__ uint32_t mnmajor_offset(uint32_t n, uint32_t k) {
    return (n >> 3) * (kRows * 16u) + (k >> 3) * 128u + (k & 7u) * 16u + (n & 7u) * 2u;
}

// Columns [c0, c0 + 16) of row r of H (tensor memory) -> MN-major B operand.
__device__ __forceinline__ void store_b_from_h(uint8_t* smem, int r, int c0, uint32_t taddr_h) {
    float v[16];
    tc::tmem_ld16(taddr_h + c0, v);
    tc::tmem_wait_ld();
#pragma unroll
    for (int h8 = 0; h8 < 16; h8 += 8) {
        __nv_bfloat16 h[8], l[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) split_bf16(v[h8 + j], h[j], l[j]);
        const uint32_t off = mnmajor_offset(c0 + h8, r);
        *reinterpret_cast<uint4*>(smem + kOffBHi + off) =
            make_uint4(pack2(h[0], h[1]), pack2(h[2], h[3]), pack2(h[4], h[5]), pack2(h[6], h[7]));
        *reinterpret_cast<uint4*>(smem + kOffBLo + off) =
            make_uint4(pack2(l[0], l[1]), pack2(l[2], l[3]), pack2(l[4], l[5]), pack2(l[6], l[7]));
    }
}

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double total = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) total += red[w];
    return total;
}

__global__ void __launch_bounds__(kThreads, 1) loss_gradient_tc_kernel(const float* __restrict__ image,
                                                                       const uint8_t* __restrict__ target_arg,
                                                                       const StepFrame* __restrict__ frame,
                                                                       float* __restrict__ grad, int width,
                                                                       int height, double* __restrict__ sums,
                                                                       int* __restrict__ status) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ double red[kThreads / 32];
    const uint8_t* __restrict__ target = frame ? frame->target : target_arg;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // thread = (block row r, column group q); warp w reads tensor-memory lanes
    // 32 (w % 4) .. 32 (w % 4) + 31, which is why rows follow w % 4
    const int r = (warp & 3) * 32 + lane;
    const int q = warp >> 2;
    const int c0 = q * kGroupCols;

    // Toeplitz operands, hi and lo parts: Wv[r'][r] = w[r - r' + 5] (A of the
    // vertical pass, K-major over r), Wh^T[c'][c] = w[c - c' + 5] (B of the
    // horizontal pass, K-major over c).
    for (int i = t; i < kRows * kRows; i += kThreads) {
        const int m = i / kRows, k = i % kRows, d = k - m + 5;
        const float w = d >= 0 && d <= 10 ? c_window_tc[d] : 0.0f;
        __nv_bfloat16 h, l;
        split_bf16(w, h, l);
        const uint32_t off = tc::kmajor_offset(m, k, kRows);
        *reinterpret_cast<__nv_bfloat16*>(smem + kOffWvHi + off) = h;
        *reinterpret_cast<__nv_bfloat16*>(smem + kOffWvLo + off) = l;
    }
    for (int i = t; i < kCols * kCols; i += kThreads) {
        const int n = i / kCols, k = i % kCols, d = k - n + 5;
        const float w = d >= 0 && d <= 10 ? c_window_tc[d] : 0.0f;
        __nv_bfloat16 h, l;
        split_bf16(w, h, l);
        const uint32_t off = tc::kmajor_offset(n, k, kCols);
        *reinterpret_cast<__nv_bfloat16*>(smem + kOffWhHi + off) = h;
        *reinterpret_cast<__nv_bfloat16*>(smem + kOffWhLo + off) = l;
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kTmemCols);
        tc::tmem_relinquish();
    }
    if (t == 0) tc::mbar_init(&bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t lane_addr = tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16);
    Sync sync{&bar, 0u, true};

    float* raw_i = reinterpret_cast<float*>(smem + kOffRawI);
    float* raw_t = reinterpret_cast<float*>(smem + kOffRawT);
    const int blocks_x = (width + kOutCols - 1) / kOutCols;
    const int blocks_y = (height + kOutRows - 1) / kOutRows;
    const int items = blocks_x * blocks_y * 3;
    const float norm = 1.0f / (3.0f * static_cast<float>(width) * height);
    double l1_sum = 0.0, sq_sum = 0.0, ssim_sum = 0.0;

#pragma unroll 1
    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        if (!sync.ok) break;  // a tensor-core pass timed out: report it, issue nothing more
        const int ch = item % 3;
        const int blk = item / 3;
        const int oy = (blk / blocks_x) * kOutRows - 10;
        const int ox = (blk % blocks_x) * kOutCols - 10;
        __syncthreads();  // the previous item's readers of the raw tiles are done
        {
            // 16 loads of each plane in flight per thread
            float vi[16], vt[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int i = j * kThreads + t;
                const int y = oy + i / kCols, x = ox + i % kCols;
                const bool in = y >= 0 && x >= 0 && y < height && x < width;
                const int64_t k = (static_cast<int64_t>(y) * width + x) * 3 + ch;
                vi[j] = in ? image[k] : 0.0f;
                vt[j] = in ? target[k] * (1.0f / 255.0f) : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int i = j * kThreads + t;
                raw_i[(i / kCols) * kRawStride + i % kCols] = vi[j];
                raw_t[(i / kCols) * kRawStride + i % kCols] = vt[j];
            }
        }
        __syncthreads();
        const float* my_i = raw_i + r * kRawStride + c0;
        const float* my_t = raw_t + r * kRawStride + c0;

        // ---- five moments: x, y, x^2, y^2, xy (x = image, y = target).
        // Pipeline: the vertical pass of map m runs on the tensor core while the
        // CUDA cores stage map m + 1; one commit covers H(m + 1) and V(m).
        auto stage_moment = [&](int m) {
            float v[kGroupCols];
#pragma unroll
            for (int c = 0; c < kGroupCols; ++c) {
                const float a = my_i[c], b = my_t[c];
                v[c] = m == 0 ? a : m == 1 ? b : m == 2 ? a * a : m == 3 ? b * b : a * b;
            }
            store_a(smem, r, c0, v);
        };
        stage_moment(0);
#pragma unroll 1
        for (int m = 0; m < 5; ++m) {
            issue(sync, [&] { issue_horizontal(smem, tmem + kColH); });
            commit_wait(sync);
            store_b_from_h(smem, r, c0, lane_addr + kColH);
            issue(sync, [&] { issue_vertical(smem, tmem + kColMoments + m * kCols); });
            if (m < 4) stage_moment(m + 1);
        }
        commit_wait(sync);

        // ---- SSIM partials at the valid centres, back-filtered one at a time;
        // the gradient of this thread's columns accumulates in registers
        const int y = oy + r;
        const bool row_centre = r >= 5 && r < kRows - 5 && y >= 0 && y < height;
        const bool row_own = r >= 10 && r < kRows - 10 && y >= 0 && y < height;
        float g[kGroupCols];
#pragma unroll
        for (int c = 0; c < kGroupCols; ++c) g[c] = 0.0f;
        auto stage_partial = [&](int p) {
            float M[5][16];
#pragma unroll
            for (int mm = 0; mm < 5; ++mm) tc::tmem_ld16(lane_addr + kColMoments + mm * kCols + c0, M[mm]);
            tc::tmem_wait_ld();
            float v[kGroupCols];
#pragma unroll
            for (int j = 0; j < kGroupCols; ++j) {
                const int c = c0 + j, x = ox + c;
                float out = 0.0f;
                if (row_centre && c >= 5 && c < kCols - 5 && x >= 0 && x < width) {
                    const float mu = M[0][j], nu = M[1][j];
                    const float inv_d = 1.0f / (mu * mu + nu * nu + kC1);
                    const float inv_e = 1.0f / (M[2][j] - mu * mu + M[3][j] - nu * nu + kC2);
                    const float lum = (2 * mu * nu + kC1) * inv_d;
                    const float cs = (2 * (M[4][j] - mu * nu) + kC2) * inv_e;
                    const float dmu = 2 * (nu - mu * lum) * inv_d * cs;
                    const float pb = 2 * lum * inv_e;
                    const float pc = -lum * cs * inv_e;
                    out = p == 0 ? dmu - nu * pb - 2 * mu * pc : p == 1 ? pb : pc;
                    if (p == 0 && sums && row_own && c >= 10 && c < kCols - 10)
                        ssim_sum += static_cast<double>(lum) * static_cast<double>(cs);
                }
                v[j] = out;
            }
            store_a(smem, r, c0, v);
        };
        // F(partial p) from the vertical-pass scratch, weighted into the gradient
        auto accumulate = [&](int p) {
            float f[16];
            tc::tmem_ld16(lane_addr + kColV + c0, f);
            tc::tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < kGroupCols; ++j) {
                const float I = my_i[j], R = my_t[j];
                const float coef = p == 0 ? 1.0f : p == 1 ? R : 2.0f * I;
                g[j] += coef * f[j];
            }
        };
        stage_partial(0);
#pragma unroll 1
        for (int p = 0; p < 3; ++p) {
            issue(sync, [&] { issue_horizontal(smem, tmem + kColH); });
            commit_wait(sync);
            if (p > 0) accumulate(p - 1);  // V(p - 1) is done; V(p) reuses its columns
            store_b_from_h(smem, r, c0, lane_addr + kColH);
            issue(sync, [&] { issue_vertical(smem, tmem + kColV); });
            if (p < 2) stage_partial(p + 1);
        }
        commit_wait(sync);
        accumulate(2);
        if (row_own) {
#pragma unroll
            for (int j = 0; j < kGroupCols; ++j) {
                const int c = c0 + j, x = ox + c;
                if (c >= 10 && c < kCols - 10 && x >= 0 && x < width) {
                    const float I = my_i[j], R = my_t[j];
                    const float d = I - R;
                    const float l1 = static_cast<float>(d > 0) - static_cast<float>(d < 0);
                    grad[(static_cast<int64_t>(y) * width + x) * 3 + ch] = (0.8f * l1 - 0.2f * g[j]) * norm;
                    if (sums) {
                        const double dd = static_cast<double>(I) - static_cast<double>(R);
                        l1_sum += fabs(dd);
                        sq_sum += dd * dd;
                    }
                }
            }
        }
    }
    if (sums) {
        const double l1s = block_sum(l1_sum, red);
        const double ss = block_sum(ssim_sum, red);
        const double sq = block_sum(sq_sum, red);
        if (t == 0) {
            atomicAdd(sums + 0, l1s);
            atomicAdd(sums + 1, ss);
            atomicAdd(sums + 2, sq);
        }
    }
    if (!sync.ok && t == 0) atomicExch(status, GSN_ERR_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
}

}  // namespace

int launch_loss_gradient_tc(const float* image, const uint8_t* target, const StepFrame* frame, float* grad, int width,
                            int height, double* sums, int* status, cudaStream_t stream) {
    if (width <= 0 || height <= 0 || !status) return GSN_ERR_INVALID_ARGUMENT;
    if (sums && cudaMemsetAsync(sums, 0, 3 * sizeof(double), stream) != cudaSuccess) return GSN_ERR_CUDA;
    // per-device launch set-up, once per device; host threads calling on the
    // same device serialise on the lock
    static std::mutex mutex;
    static bool configured[64] = {};
    static int sm_count[64] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return GSN_ERR_CUDA;
    int sms = 0;
    {
        std::lock_guard<std::mutex> lock(mutex);
        if (!configured[device]) {
            if (cudaFuncSetAttribute(loss_gradient_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kSmemBytes)) != cudaSuccess ||
                cudaDeviceGetAttribute(&sm_count[device], cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
                return GSN_ERR_CUDA;
            configured[device] = true;
        }
        sms = sm_count[device];
    }
    const int items = ((width + kOutCols - 1) / kOutCols) * ((height + kOutRows - 1) / kOutRows) * 3;
    const int grid = items < sms ? items : sms;
    loss_gradient_tc_kernel<<<grid, kThreads, kSmemBytes, stream>>>(image, target, frame, grad, width, height, sums,
                                                               status);
    return launched(1);
}

}  // namespace gsn
