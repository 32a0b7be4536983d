// Test-infrastructure harness: the reference's LBVH 3-NN (src/core/knn/knn.cu,
// compiled unmodified from the reference tree) behind extern "C". Not part of
// the product.
#include "core/knn/knn.cu"

extern "C" {

// ComputeMeanDist2Cuda (knn.cu:180-255) on host xyz triples.
int ref_knn_mean_dist2(const float* points, int count, float* out) {
    std::vector<Eigen::Vector3f> p(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i) p[i] = Eigen::Vector3f(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    std::vector<float> r = gs_native::ComputeMeanDist2Cuda(p);
    if (r.size() != p.size()) return -1;
    for (int i = 0; i < count; ++i) out[i] = r[i];
    return 0;
}

}  // extern "C"
