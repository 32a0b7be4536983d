// Drop-in ComputeMeanDist2Cuda (reference: src/core/knn/knn.h:9, knn.cu:180-255):
// for every point the mean of its (up to) three smallest squared distances to
// the other points (0 for fewer than two points), in input order; an empty
// vector signals failure, like the reference.
//
// The reference takes std::vector<Eigen::Vector3f>; this header accepts any
// element type holding three contiguous floats (Eigen::Vector3f included), so it
// needs no Eigen itself.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

namespace gs_native {

// Host xyz triples in, host results out; optional neighbour indices (3 per point,
// -1 when missing). Returns false on any CUDA failure.
bool ComputeMeanDist2(const float* xyz, int count, float* mean_dist2, int* neighbors = nullptr,
                      cudaStream_t stream = nullptr);

template <class Vec3>
std::vector<float> ComputeMeanDist2Cuda(const std::vector<Vec3>& points) {
    static_assert(sizeof(Vec3) == 3 * sizeof(float), "points must hold three contiguous floats");
    std::vector<float> result(points.size(), 0.0f);
    if (points.size() > static_cast<size_t>(0x7fffffff)) return {};
    if (points.size() < 2) return result;
    if (!ComputeMeanDist2(reinterpret_cast<const float*>(points.data()), static_cast<int>(points.size()),
                          result.data()))
        return {};
    return result;
}

}  // namespace gs_native
