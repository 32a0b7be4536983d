// LBVH 3-NN launcher (knn.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace gsn {

// Byte offsets of the sub-buffers of the KNN workspace for n points.
struct KnnLayout {
    int leaves;
    size_t bounds, keys, keys_alt, ids, ids_alt, lo, hi, status, sort, total;
};
KnnLayout knn_layout(int n);

// points: device float[3 n] (xyz); mean_dist2: device float[n]; neighbors:
// optional device int[3 n] (-1 when missing); workspace: knn_layout(n).total bytes.
int launch_knn3(const float* points, int n, float* mean_dist2, int* neighbors, void* workspace, cudaStream_t s);

}  // namespace gsn
