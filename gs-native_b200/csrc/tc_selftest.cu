// Self-test of the tcgen05 building blocks (tcgen05.cuh): one CTA computes
// D (128 x 64, fp32) = A (128 x 128) * B^T (B: 64 x 128) with bf16 operands
// staged in shared memory in the canonical K-major layout, the product
// accumulated in tensor memory over eight K = 16 MMAs and read back with
// tcgen05.ld. The SSIM filter GEMMs of the precision form use exactly these
// descriptors and instruction forms; the test pins them against a CPU product.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"
#include "tcgen05.cuh"

namespace gsn {

namespace {

constexpr int kM = 128, kN = 64, kK = 128;
constexpr size_t kSelftestSmem = (kM + kN) * kK * sizeof(__nv_bfloat16);  // 48 KB
constexpr long long kWaitCycles = 2000000000LL;

__global__ void __launch_bounds__(128) tc_gemm_selftest_kernel(const float* __restrict__ a,
                                                               const float* __restrict__ b, float* __restrict__ d,
                                                               int* __restrict__ status) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    uint8_t* sa = smem;
    uint8_t* sb = smem + kM * kK * sizeof(__nv_bfloat16);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    for (int i = t; i < kM * kK; i += 128)
        *reinterpret_cast<__nv_bfloat16*>(sa + tc::kmajor_offset(i / kK, i % kK, kK)) = __float2bfloat16_rn(a[i]);
    for (int i = t; i < kN * kK; i += 128)
        *reinterpret_cast<__nv_bfloat16*>(sb + tc::kmajor_offset(i / kK, i % kK, kK)) = __float2bfloat16_rn(b[i]);
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kN);
        tc::tmem_relinquish();
    }
    if (t == 0) tc::mbar_init(&bar, 1);
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    if (t == 0) {
        const uint32_t idesc = tc::idesc_bf16_f32(kM, kN);
        const uint32_t base_a = tc::smem_u32(sa), base_b = tc::smem_u32(sb);
#pragma unroll 1
        for (int k = 0; k < kK / 16; ++k) {
            // K = 16 step k starts at core-matrix column 2k (256 bytes per step)
            const uint64_t da = tc::smem_desc(base_a + k * 256, 128, kK * 16);
            const uint64_t db = tc::smem_desc(base_b + k * 256, 128, kK * 16);
            tc::mma_bf16(tmem, da, db, idesc, k > 0);
        }
        tc::commit(&bar);
    }
    const bool ok = __syncthreads_and(tc::mbar_wait(&bar, 0, kWaitCycles));
    tc::fence_after_sync();
    if (ok) {
#pragma unroll 1
        for (int c = 0; c < kN; c += 16) {
            float v[16];
            tc::tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c, v);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) d[(warp * 32 + lane) * kN + c + i] = v[i];
        }
    } else {
        if (t == 0) atomicExch(status, GSN_ERR_TIMEOUT);
        tc::mbar_wait(&bar, 0, kWaitCycles);  // let the MMAs drain before freeing
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kN);
}

}  // namespace

int launch_tc_gemm_selftest(const float* a, const float* b, float* d, int* status, cudaStream_t stream) {
    if (!a || !b || !d || !status) return GSN_ERR_INVALID_ARGUMENT;
    if (cudaFuncSetAttribute(tc_gemm_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kSelftestSmem)) != cudaSuccess)
        return GSN_ERR_CUDA;
    tc_gemm_selftest_kernel<<<1, 128, kSelftestSmem, stream>>>(a, b, d, status);
    return launched(1);
}

}  // namespace gsn
