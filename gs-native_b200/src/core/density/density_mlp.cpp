// gs_native::DensityMlp over the kernels of csrc/mlp.cu.
#include "core/density/density_mlp.h"

#include <cmath>
#include <random>

#include "gsn_types.h"
#include "mlp.h"

namespace gs_native {

static_assert(DensityMlp::kParams == gsn::kMlpParams, "MLP weight count");

bool DensityMlp::Ready() {
    if (master_.get()) return true;
    return master_.Reserve(kParams) && m_.Reserve(kParams) && v_.Reserve(kParams) && grad_.Reserve(kParams) &&
           half_.Reserve(kParams) && loss_.Reserve(1);
}

bool DensityMlp::Initialize(uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::vector<float> w(kParams, 0.0f);
    auto fill = [&](int offset, int rows, int cols) {
        std::normal_distribution<float> n(0.0f, std::sqrt(2.0f / cols));
        for (int i = 0; i < rows * cols; ++i) w[offset + i] = n(rng);
    };
    fill(0, 64, 16);           // W1
    fill(1024 + 64, 64, 64);   // W2
    fill(5184 + 64, 4, 64);    // W3
    return SetWeights(w.data());
}

bool DensityMlp::SetWeights(const float* host) {
    if (!host || !Ready()) return false;
    step_ = 0;
    return cudaMemcpyAsync(master_.get(), host, kParams * sizeof(float), cudaMemcpyHostToDevice, stream_) ==
               cudaSuccess &&
           cudaMemsetAsync(m_.get(), 0, kParams * sizeof(float), stream_) == cudaSuccess &&
           cudaMemsetAsync(v_.get(), 0, kParams * sizeof(float), stream_) == cudaSuccess &&
           cudaMemsetAsync(grad_.get(), 0, kParams * sizeof(float), stream_) == cudaSuccess &&
           gsn::launch_mlp_to_half(master_.get(), half_.get(), stream_) == GSN_OK &&
           cudaStreamSynchronize(stream_) == cudaSuccess;
}

bool DensityMlp::GetWeights(float* host) const {
    if (!host || !master_.get()) return false;
    return cudaMemcpyAsync(host, master_.get(), kParams * sizeof(float), cudaMemcpyDeviceToHost, stream_) ==
               cudaSuccess &&
           cudaStreamSynchronize(stream_) == cudaSuccess;
}

double DensityMlp::WeightSum(const float* weights, int n) {
    std::vector<float> w(static_cast<size_t>(n));
    if (cudaMemcpyAsync(w.data(), weights, w.size() * sizeof(float), cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
        return -1.0;
    double s = 0.0;
    for (float x : w) s += x;
    return s;
}

bool DensityMlp::Gradients(const float* features, const int* labels, const float* weights, int n, float* grad_host,
                           double* loss) {
    if (!features || !labels || !weights || n <= 0 || !grad_host || !Ready()) return false;
    const double total = WeightSum(weights, n);
    if (!(total > 0.0)) return false;
    if (cudaMemsetAsync(grad_.get(), 0, kParams * sizeof(float), stream_) != cudaSuccess ||
        cudaMemsetAsync(loss_.get(), 0, sizeof(double), stream_) != cudaSuccess ||
        gsn::launch_mlp_gradients(features, labels, weights, n, static_cast<float>(1.0 / total), half_.get(),
                                  grad_.get(), loss_.get(), stream_) != GSN_OK ||
        cudaMemcpyAsync(grad_host, grad_.get(), kParams * sizeof(float), cudaMemcpyDeviceToHost, stream_) !=
            cudaSuccess)
        return false;
    double l = 0.0;
    if (cudaMemcpyAsync(&l, loss_.get(), sizeof(double), cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
        return false;
    if (loss) *loss = l;
    return cudaMemsetAsync(grad_.get(), 0, kParams * sizeof(float), stream_) == cudaSuccess;
}

bool DensityMlp::Train(const float* features, const int* labels, const float* weights, int n, int steps, float lr,
                       double* loss) {
    if (!features || !labels || !weights || n <= 0 || steps < 0 || !(lr > 0.0f) || !Ready()) return false;
    const double total = WeightSum(weights, n);
    if (!(total > 0.0)) return false;
    const float norm = static_cast<float>(1.0 / total);
    for (int k = 0; k < steps; ++k) {
        const bool last = k + 1 == steps;
        if (last && cudaMemsetAsync(loss_.get(), 0, sizeof(double), stream_) != cudaSuccess) return false;
        if (gsn::launch_mlp_gradients(features, labels, weights, n, norm, half_.get(), grad_.get(),
                                      last ? loss_.get() : nullptr, stream_) != GSN_OK)
            return false;
        ++step_;
        const float c1 = static_cast<float>(1.0 / (1.0 - std::pow(0.9, static_cast<double>(step_))));
        const float c2 = static_cast<float>(1.0 / (1.0 - std::pow(0.999, static_cast<double>(step_))));
        if (gsn::launch_mlp_adam(master_.get(), m_.get(), v_.get(), grad_.get(), half_.get(), lr, c1, c2, stream_) !=
            GSN_OK)
            return false;
    }
    double l = 0.0;
    if (steps > 0 &&
        cudaMemcpyAsync(&l, loss_.get(), sizeof(double), cudaMemcpyDeviceToHost, stream_) != cudaSuccess)
        return false;
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return false;
    if (loss) *loss = l;
    return true;
}

bool DensityMlp::Infer(const float* features, int n, float confidence, int8_t* actions, float* probs) {
    if (n == 0) return true;
    if (!features || n < 0 || !actions || !master_.get()) return false;
    return gsn::launch_mlp_infer(features, n, half_.get(), confidence, actions, probs, stream_) == GSN_OK;
}

}  // namespace gs_native
