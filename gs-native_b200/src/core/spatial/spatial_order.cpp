// gs_native::SpatialOrder over the Morton-key, sort and gather kernels.
#include "core/spatial/spatial_order.h"

#include <algorithm>

#include "kernels.h"

namespace gs_native {

bool SpatialOrder::Compute(const float* params, int count) {
    if (!params || count <= 0) return false;
    const size_t n = static_cast<size_t>(count);
    if (!keys_[0].Reserve(n) || !keys_[1].Reserve(n) || !ids_[0].Reserve(n) || !ids_[1].Reserve(n) ||
        !bounds_.Reserve(6) || !sort_scratch_.Reserve(gsn::radix_sort_scratch_bytes(count)))
        return false;
    if (gsn::launch_morton_keys(params, count, bounds_.get(), keys_[0].get(), stream_) != GSN_OK) return false;
    bool in_alt = false;
    const gsn::RadixSortScratch scratch = gsn::radix_sort_scratch(sort_scratch_.get(), count);
    if (gsn::launch_radix_sort(keys_[0].get(), ids_[0].get(), keys_[1].get(), ids_[1].get(), true, count, nullptr,
                               0, 30, scratch, &in_alt, stream_) != GSN_OK)
        return false;
    perm_ = ids_[in_alt ? 1 : 0].get();
    count_ = count;
    return true;
}

bool SpatialOrder::Apply(float* params, int count, bool bf16_sh, const int* parents) {
    if (!params || count != count_ || !perm_) return false;
    const size_t floats = static_cast<size_t>(count) * (bf16_sh ? GSN_SH_INDEX + 24 : GSN_PARAM_COUNT);
    if (!block_.Reserve(floats) || !parents_.Reserve(static_cast<size_t>(count))) return false;
    if (gsn::launch_gather_gaussians(params, block_.get(), perm_, count, bf16_sh, stream_) != GSN_OK ||
        cudaMemcpyAsync(params, block_.get(), floats * sizeof(float), cudaMemcpyDeviceToDevice, stream_) !=
            cudaSuccess ||
        gsn::launch_compose_parents(parents, perm_, count, parents_.get(), stream_) != GSN_OK)
        return false;
    return true;
}

bool SpatialOrder::Compose(const int* parents, int* out) {
    if (!out || !perm_) return false;
    return gsn::launch_compose_parents(parents, perm_, count_, out, stream_) == GSN_OK;
}

}  // namespace gs_native
