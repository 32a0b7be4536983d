// Learned density policy (gs-native extension; the reference has only the
// threshold rule of density_controller.cu:60-116): a 16 -> 64 -> 64 -> 4 MLP
// over per-Gaussian statistics proposing keep / clone / split / prune, with
// fp16 working weights and fp32 arithmetic, trained on the GPU by the kernels
// of csrc/mlp.cu (full-batch Adam on weighted cross-entropy).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "util/device_array.h"

namespace gs_native {

class DensityMlp {
public:
    static constexpr int kParams = 5508;

    // He-initialised weights from a seed (host), Adam state cleared.
    bool Initialize(uint64_t seed);
    bool SetWeights(const float* host);  // kParams floats
    bool GetWeights(float* host) const;
    void SetStream(cudaStream_t stream) { stream_ = stream; }

    // Gradient (host, kParams floats) and loss of the mean weighted cross-entropy
    // of n device samples (features [n][16], labels [n] in 0..3, weights [n]).
    bool Gradients(const float* features, const int* labels, const float* weights, int n, float* grad_host,
                   double* loss);
    // `steps` full-batch Adam steps at learning rate lr; *loss = the loss
    // before the last step.
    bool Train(const float* features, const int* labels, const float* weights, int n, int steps, float lr,
               double* loss);
    // Actions of n device feature rows: argmax where its probability >= confidence, else -1.
    bool Infer(const float* features, int n, float confidence, int8_t* actions, float* probs = nullptr);
    const void* WeightsF16() const { return half_.get(); }

private:
    bool Ready();
    double WeightSum(const float* weights, int n);

    cudaStream_t stream_ = nullptr;
    DeviceArray<float> master_, m_, v_, grad_;
    DeviceArray<uint16_t> half_;
    DeviceArray<double> loss_;
    uint64_t step_ = 0;
};

}  // namespace gs_native
