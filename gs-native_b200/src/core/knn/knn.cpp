// Host side of the LBVH 3-NN drop-in (see knn.h).
#include "core/knn/knn.h"

#include "knn_kernels.h"
#include "util/device_array.h"

namespace gs_native {

bool ComputeMeanDist2(const float* xyz, int count, float* mean_dist2, int* neighbors, cudaStream_t stream) {
    if (count < 0 || (count > 0 && (!xyz || !mean_dist2))) return false;
    if (count == 0) return true;
    const size_t n = static_cast<size_t>(count);
    DeviceArray<float> points, dist;
    DeviceArray<int> nb;
    DeviceArray<unsigned char> work;
    if (!points.Reserve(3 * n) || !dist.Reserve(n) || (neighbors && !nb.Reserve(3 * n)) ||
        !work.Reserve(gsn::knn_layout(count).total))
        return false;
    if (cudaMemcpyAsync(points.get(), xyz, 3 * n * sizeof(float), cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return false;
    if (gsn::launch_knn3(points.get(), count, dist.get(), neighbors ? nb.get() : nullptr, work.get(), stream) != 0)
        return false;
    if (cudaMemcpyAsync(mean_dist2, dist.get(), n * sizeof(float), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        return false;
    if (neighbors &&
        cudaMemcpyAsync(neighbors, nb.get(), 3 * n * sizeof(int), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        return false;
    return cudaStreamSynchronize(stream) == cudaSuccess;
}

}  // namespace gs_native
