// Launchers of the learned density policy's MLP kernels (mlp.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gsn {

// 16 -> 64 -> 64 -> 4 weights, flat: W1[64][16], b1[64], W2[64][64], b2[64], W3[4][64], b3[4].
constexpr int kMlpParams = 64 * 16 + 64 + 64 * 64 + 64 + 4 * 64 + 4;  // 5508

// actions[i] = argmax of the softmax if its probability >= confidence, else -1
// (the plain rule decides); probs (optional) [n][4].
int launch_mlp_infer(const float* features, int n, const void* weights_f16, float confidence, int8_t* actions,
                     float* probs, cudaStream_t stream);
// Accumulates into grad the gradient of sum_i weight_norm * w_i * CE(softmax(MLP(f_i)), label_i)
// and, when loss is given, adds that loss to *loss (FP64).
int launch_mlp_gradients(const float* features, const int* labels, const float* sample_weights, int n,
                         float weight_norm, const void* weights_f16, float* grad, double* loss, cudaStream_t stream);
// Adam step of the fp32 master weights (lr, bias corrections c1, c2); writes the
// fp16 copy and clears grad.
int launch_mlp_adam(float* master, float* m, float* v, float* grad, void* weights_f16, float lr, float c1, float c2,
                    cudaStream_t stream);
int launch_mlp_to_half(const float* master, void* weights_f16, cudaStream_t stream);

}  // namespace gsn
