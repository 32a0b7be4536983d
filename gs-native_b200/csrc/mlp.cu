// Learned density policy: a 16 -> 64 -> 64 -> 4 MLP (ReLU, softmax over
// keep / clone / split / prune) with fp16 working weights and fp32 arithmetic.
//
// Weights, flat (kMlpParams floats): W1[64][16], b1[64], W2[64][64], b2[64],
// W3[4][64], b3[4]. Training keeps an fp32 master copy and Adam moments; the
// forward and backward passes read the fp16 copy (mixed precision).
//
// Training step (fused): a CTA takes a tile of 128 samples, one thread per
// sample runs the forward and backward passes and leaves its activations and
// deltas in shared memory; the CTA then forms the tile's weight gradients as
// small GEMMs over the tile (each thread a set of entries) and adds them to the
// global fp32 gradient with one atomic per entry.
#include <cuda_fp16.h>

#include "common.cuh"
#include "mlp.h"

namespace gsn {

namespace {

constexpr int kIn = 16, kHid = 64, kOut = 4;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kOut * kHid;
static_assert(kOffB3 + kOut == kMlpParams, "weight layout");

constexpr int kSampleTile = 128;       // samples per training CTA
constexpr int kVec = kHid + 1;   // padded shared row of a per-sample vector

__device__ __forceinline__ float w(const __half* W, int i) { return __half2float(W[i]); }

__global__ void __launch_bounds__(256) mlp_infer_kernel(const float* __restrict__ features, int n,
                                                        const __half* __restrict__ weights, float confidence,
                                                        int8_t* __restrict__ actions, float* __restrict__ probs) {
    __shared__ __half W[kMlpParams];
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) W[i] = weights[i];
    __syncthreads();
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    float f[kIn];
    const float4* fp = reinterpret_cast<const float4*>(features + static_cast<int64_t>(id) * kIn);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 v = fp[q];
        f[4 * q] = v.x;
        f[4 * q + 1] = v.y;
        f[4 * q + 2] = v.z;
        f[4 * q + 3] = v.w;
    }
    float h1[kHid];
#pragma unroll
    for (int o = 0; o < kHid; ++o) {
        float acc = w(W, kOffB1 + o);
#pragma unroll
        for (int k = 0; k < kIn; ++k) acc += w(W, kOffW1 + o * kIn + k) * f[k];
        h1[o] = fmaxf(acc, 0.0f);
    }
    float logit[kOut];
#pragma unroll
    for (int a = 0; a < kOut; ++a) logit[a] = w(W, kOffB3 + a);
#pragma unroll 4
    for (int o = 0; o < kHid; ++o) {
        float acc = w(W, kOffB2 + o);
#pragma unroll
        for (int k = 0; k < kHid; ++k) acc += w(W, kOffW2 + o * kHid + k) * h1[k];
        const float h = fmaxf(acc, 0.0f);
#pragma unroll
        for (int a = 0; a < kOut; ++a) logit[a] += w(W, kOffW3 + a * kHid + o) * h;
    }
    float mx = logit[0];
    int best = 0;
#pragma unroll
    for (int a = 1; a < kOut; ++a)
        if (logit[a] > mx) {
            mx = logit[a];
            best = a;
        }
    float e[kOut], sum = 0.0f;
#pragma unroll
    for (int a = 0; a < kOut; ++a) {
        e[a] = __expf(logit[a] - mx);
        sum += e[a];
    }
    if (probs) {
#pragma unroll
        for (int a = 0; a < kOut; ++a) probs[static_cast<int64_t>(id) * kOut + a] = e[a] / sum;
    }
    actions[id] = e[best] / sum >= confidence ? static_cast<int8_t>(best) : static_cast<int8_t>(-1);
}

__global__ void __launch_bounds__(kSampleTile) mlp_train_kernel(const float* __restrict__ features,
                                                          const int* __restrict__ labels,
                                                          const float* __restrict__ sample_weights, int n,
                                                          float weight_norm, const __half* __restrict__ weights,
                                                          float* __restrict__ grad, double* __restrict__ loss) {
    extern __shared__ float sm[];
    __shared__ __half W[kMlpParams];
    float* sf = sm;                        // [kSampleTile][kIn]
    float* sh1 = sf + kSampleTile * kIn;         // [kSampleTile][kVec]
    float* sh2 = sh1 + kSampleTile * kVec;
    float* sdz1 = sh2 + kSampleTile * kVec;
    float* sdz2 = sdz1 + kSampleTile * kVec;
    float* sdl = sdz2 + kSampleTile * kVec;      // [kSampleTile][kOut]
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) W[i] = weights[i];
    __syncthreads();
    const int s = threadIdx.x;
    const int id = blockIdx.x * kSampleTile + s;
    const bool live = id < n;
    float f[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) f[k] = live ? features[static_cast<int64_t>(id) * kIn + k] : 0.0f;
    const int label = live ? labels[id] : 0;
    const float sw = live ? sample_weights[id] * weight_norm : 0.0f;
    // forward
    float* h1 = sh1 + s * kVec;
    float* h2 = sh2 + s * kVec;
#pragma unroll 4
    for (int o = 0; o < kHid; ++o) {
        float acc = w(W, kOffB1 + o);
#pragma unroll
        for (int k = 0; k < kIn; ++k) acc += w(W, kOffW1 + o * kIn + k) * f[k];
        h1[o] = fmaxf(acc, 0.0f);
    }
    float logit[kOut];
#pragma unroll
    for (int a = 0; a < kOut; ++a) logit[a] = w(W, kOffB3 + a);
#pragma unroll 2
    for (int o = 0; o < kHid; ++o) {
        float acc = w(W, kOffB2 + o);
#pragma unroll 8
        for (int k = 0; k < kHid; ++k) acc += w(W, kOffW2 + o * kHid + k) * h1[k];
        const float h = fmaxf(acc, 0.0f);
        h2[o] = h;
#pragma unroll
        for (int a = 0; a < kOut; ++a) logit[a] += w(W, kOffW3 + a * kHid + o) * h;
    }
    // softmax cross-entropy, weighted and normalised by the batch weight
    float mx = fmaxf(fmaxf(logit[0], logit[1]), fmaxf(logit[2], logit[3]));
    float e[kOut], sum = 0.0f;
#pragma unroll
    for (int a = 0; a < kOut; ++a) {
        e[a] = expf(logit[a] - mx);
        sum += e[a];
    }
    float dl[kOut];
#pragma unroll
    for (int a = 0; a < kOut; ++a) {
        const float p = e[a] / sum;
        dl[a] = sw * (p - (a == label ? 1.0f : 0.0f));
        sdl[s * kOut + a] = dl[a];
    }
    if (live && loss) {
        const double lp = static_cast<double>(logit[label] - mx) - log(static_cast<double>(sum));
        atomicAdd(loss, -static_cast<double>(sw) * lp);
    }
    // backward through layer 3 and the second ReLU
    float* dz2 = sdz2 + s * kVec;
#pragma unroll 4
    for (int o = 0; o < kHid; ++o) {
        float d = 0.0f;
#pragma unroll
        for (int a = 0; a < kOut; ++a) d += w(W, kOffW3 + a * kHid + o) * dl[a];
        dz2[o] = h2[o] > 0.0f ? d : 0.0f;
    }
    // backward through layer 2 and the first ReLU
    float* dz1 = sdz1 + s * kVec;
#pragma unroll 2
    for (int k = 0; k < kHid; ++k) {
        float d = 0.0f;
#pragma unroll 8
        for (int o = 0; o < kHid; ++o) d += w(W, kOffW2 + o * kHid + k) * dz2[o];
        dz1[k] = h1[k] > 0.0f ? d : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < kIn; ++k) sf[s * kIn + k] = f[k];
    __syncthreads();
    // weight gradients of the tile: each thread a set of entries, summed over samples
    for (int e2 = threadIdx.x; e2 < kMlpParams; e2 += kSampleTile) {
        float acc = 0.0f;
        if (e2 < kOffB1) {
            const int o = e2 / kIn, k = e2 % kIn;
            for (int q = 0; q < kSampleTile; ++q) acc += sdz1[q * kVec + o] * sf[q * kIn + k];
        } else if (e2 < kOffW2) {
            const int o = e2 - kOffB1;
            for (int q = 0; q < kSampleTile; ++q) acc += sdz1[q * kVec + o];
        } else if (e2 < kOffB2) {
            const int o = (e2 - kOffW2) / kHid, k = (e2 - kOffW2) % kHid;
            for (int q = 0; q < kSampleTile; ++q) acc += sdz2[q * kVec + o] * sh1[q * kVec + k];
        } else if (e2 < kOffW3) {
            const int o = e2 - kOffB2;
            for (int q = 0; q < kSampleTile; ++q) acc += sdz2[q * kVec + o];
        } else if (e2 < kOffB3) {
            const int a = (e2 - kOffW3) / kHid, o = (e2 - kOffW3) % kHid;
            for (int q = 0; q < kSampleTile; ++q) acc += sdl[q * kOut + a] * sh2[q * kVec + o];
        } else {
            const int a = e2 - kOffB3;
            for (int q = 0; q < kSampleTile; ++q) acc += sdl[q * kOut + a];
        }
        if (acc != 0.0f) atomicAdd(grad + e2, acc);
    }
}

// Adam on the fp32 master weights; refreshes the fp16 working copy and clears
// the gradient for the next step.
__global__ void mlp_adam_kernel(float* __restrict__ master, float* __restrict__ m, float* __restrict__ v,
                                float* __restrict__ grad, __half* __restrict__ weights, float lr, float c1,
                                float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const float g = grad[i];
    const float mi = 0.9f * m[i] + 0.1f * g;
    const float vi = 0.999f * v[i] + 0.001f * g * g;
    m[i] = mi;
    v[i] = vi;
    const float p = master[i] - lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
    master[i] = p;
    weights[i] = __float2half_rn(p);
    grad[i] = 0.0f;
}

__global__ void mlp_to_half_kernel(const float* __restrict__ master, __half* __restrict__ weights) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kMlpParams) weights[i] = __float2half_rn(master[i]);
}

constexpr size_t kTrainSmem = sizeof(float) * (kSampleTile * kIn + 4 * kSampleTile * kVec + kSampleTile * kOut);

}  // namespace

int launch_mlp_infer(const float* features, int n, const void* weights_f16, float confidence, int8_t* actions,
                     float* probs, cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    mlp_infer_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(features, n, static_cast<const __half*>(weights_f16),
                                                           confidence, actions, probs);
    return launched(1);
}

int launch_mlp_gradients(const float* features, const int* labels, const float* sample_weights, int n,
                         float weight_norm, const void* weights_f16, float* grad, double* loss, cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    static bool configured[64] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return GSN_ERR_CUDA;
    if (!configured[device]) {
        if (cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kTrainSmem)) != cudaSuccess)
            return GSN_ERR_CUDA;
        configured[device] = true;
    }
    mlp_train_kernel<<<ceil_div(n, kSampleTile), kSampleTile, kTrainSmem, stream>>>(
        features, labels, sample_weights, n, weight_norm, static_cast<const __half*>(weights_f16), grad, loss);
    return launched(1);
}

int launch_mlp_adam(float* master, float* m, float* v, float* grad, void* weights_f16, float lr, float c1, float c2,
                    cudaStream_t stream) {
    mlp_adam_kernel<<<ceil_div(kMlpParams, 256), 256, 0, stream>>>(master, m, v, grad,
                                                                     static_cast<__half*>(weights_f16), lr, c1, c2);
    return launched(1);
}

int launch_mlp_to_half(const float* master, void* weights_f16, cudaStream_t stream) {
    mlp_to_half_kernel<<<ceil_div(kMlpParams, 256), 256, 0, stream>>>(master, static_cast<__half*>(weights_f16));
    return launched(1);
}

}  // namespace gsn
