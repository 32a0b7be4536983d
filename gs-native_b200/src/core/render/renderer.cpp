// gs_native::Renderer over the sm_100a kernels of csrc/ (reference behaviour:
// src/core/render/renderer.cu:359-590).
#include "core/render/renderer.h"

#include <algorithm>
#include <climits>
#include <cstdint>

#include "kernels.h"
#include "profile.h"

namespace gs_native {

namespace {

int TileBits(int tile_count) {
    int bits = 0;
    for (unsigned int t = static_cast<unsigned int>(tile_count - 1); t; t >>= 1) ++bits;
    return bits;
}

}  // namespace

Renderer::Renderer() = default;

Renderer::~Renderer() {
    if (host_records_) cudaFreeHost(host_records_);
}

bool Renderer::SetRecordCapacity(int64_t records) {
    if (records < 0 || records > INT_MAX) return false;
    if (records == 0) {
        fixed_capacity_ = false;
        return true;
    }
    if (!ReserveRecords(records)) return false;
    fixed_capacity_ = true;
    return true;
}

bool Renderer::ReserveGaussians(int count) {
    size_t n = static_cast<size_t>(std::max(count, 1));
    if (n <= gaussian_capacity_ && counters_.get()) return true;
    size_t grow = std::max(n, gaussian_capacity_ + gaussian_capacity_ / 4);
    bool ok = means_.Reserve(grow) && conic_opacities_.Reserve(grow) && colors_.Reserve(grow) &&
              depths_.Reserve(grow) && radii_.Reserve(grow) && rects_.Reserve(grow) &&
              tile_counts_.Reserve(grow) && cull_counts_.Reserve(grow) && depth_keys_[0].Reserve(grow) &&
              depth_keys_[1].Reserve(grow) &&
              depth_ids_[0].Reserve(grow) && depth_ids_[1].Reserve(grow) && record_start_.Reserve(grow + 1) &&
              counters_.Reserve(3);
    if (!ok) return false;
    gaussian_capacity_ = grow;
    return true;
}

bool Renderer::ReserveRecords(int64_t records) {
    size_t r = static_cast<size_t>(std::max<int64_t>(records, 1));
    if (r <= static_cast<size_t>(record_capacity_) && tile_keys_[0].get()) return true;
    size_t grow = std::max(r, static_cast<size_t>(record_capacity_ + record_capacity_ / 2));
    grow = std::min<size_t>(grow, INT_MAX);
    if (grow < r) return false;
    bool ok = tile_keys_[0].Reserve(grow) && tile_keys_[1].Reserve(grow) && record_ids_[0].Reserve(grow) &&
              record_ids_[1].Reserve(grow) && record_warps_.Reserve(2 * (grow / 32 + 1));
    if (!ok) return false;
    record_words_ = static_cast<int64_t>(grow / 32 + 1);
    record_capacity_ = static_cast<int64_t>(grow);
    return true;
}

bool Renderer::Render(const GaussianBuffers& gaussians, const CameraParams& camera, const float* background,
                      float* image, int sh_degree) {
    const int count = gaussians.gaussian_count_;
    if (count < 0 || count == INT_MAX || (count > 0 && !gaussians.gaussians_)) return false;
    if (!background || !image || camera.width_ <= 0 || camera.height_ <= 0 || camera.tile_count_x_ <= 0 ||
        camera.tile_count_y_ <= 0)
        return false;
    const int64_t tile_count_long = static_cast<int64_t>(camera.tile_count_x_) * camera.tile_count_y_;
    if (tile_count_long >= INT_MAX) return false;
    const int tile_count = static_cast<int>(tile_count_long);
    sh_degree = std::clamp(sh_degree, 0, 3);
    if (!ReserveGaussians(count)) return false;
    if (static_cast<size_t>(tile_count) > tile_capacity_) {
        if (!tile_offsets_.Reserve(static_cast<size_t>(tile_count) + 1)) return false;
        tile_capacity_ = static_cast<size_t>(tile_count);
    }
    const size_t pixels = static_cast<size_t>(camera.width_) * camera.height_;
    if (pixels > pixel_capacity_) {
        if (!contributors_.Reserve(pixels)) return false;
        pixel_capacity_ = pixels;
    }
    if (!fixed_capacity_ && !ReserveRecords(std::max<int64_t>(record_capacity_, 1))) return false;
    const int sort_max = static_cast<int>(std::max<int64_t>(count, record_capacity_));
    if (static_cast<size_t>(sort_max) > sort_scratch_count_ || !sort_scratch_.get()) {
        size_t want = std::max<size_t>(sort_max, sort_scratch_count_ + sort_scratch_count_ / 2);
        if (!sort_scratch_.Reserve(gsn::radix_sort_scratch_bytes(static_cast<int>(std::min<size_t>(want, INT_MAX)))))
            return false;
        sort_scratch_count_ = want;
    }
    if (static_cast<size_t>(count) > scan_scratch_count_ || !scan_scratch_.get()) {
        if (!scan_scratch_.Reserve(gsn::scan_scratch_bytes(std::max(count, 1)))) return false;
        scan_scratch_count_ = static_cast<size_t>(std::max(count, 1));
    }
    if (!host_records_ && cudaMallocHost(&host_records_, sizeof(int)) != cudaSuccess) {
        host_records_ = nullptr;
        return false;
    }
    record_offsets_valid_ = false;
    last_count_ = count;
    const gsn_camera& cam = AsGsnCamera(camera);
    cudaStream_t s = stream_;
    if (cudaMemsetAsync(counters_.get(), 0, 2 * sizeof(int), s) != cudaSuccess) return false;

    int64_t records = 0;
    if (count > 0) {
        gsn::ProjectOutputs po{means_.get(), conic_opacities_.get(), colors_.get(), depths_.get(),
                               rects_.get(), tile_counts_.get(), depth_keys_[0].get(), radii_.get(),
                               exact_culling_ ? cull_counts_.get() : nullptr,
                               // the fast forms order depths on 24-bit keys (one radix pass less;
                               // depths equal to 2^-16 relative may swap their blend order)
                               fast_blend_ ? 8 : 0};
        gsn::stage_mark(s, gsn::kStageProject);
        if (gsn::launch_project(gaussians.gaussians_, count, cam, device_camera_, sh_degree, bf16_sh_, po, s) != GSN_OK) return false;
        gsn::stage_mark(s, gsn::kStageDepthSort);
        gsn::RadixSortScratch scratch = gsn::radix_sort_scratch(sort_scratch_.get(), sort_max);
        bool in_alt = false;
        // culled Gaussians (depth key 0xFFFFFFFF) leave the sort in its first
        // pass: the later passes, the record scan and the emission see only the
        // visible ones (their order - depth, then id - is unchanged)
        int* visible = counters_.get() + 2;
        if (gsn::launch_radix_sort_dropping(depth_keys_[0].get(), depth_ids_[0].get(), depth_keys_[1].get(),
                                            depth_ids_[1].get(), true, count, nullptr, 0, fast_blend_ ? 24 : 32,
                                            scratch, &in_alt, visible, s) != GSN_OK)
            return false;
        const uint32_t* by_depth = depth_ids_[in_alt ? 1 : 0].get();
        if (!OrderBySort(by_depth, visible, count, camera, tile_count, &records)) return false;
    } else {
        last_records_ = 0;
        sorted_ids_ = record_ids_[0].get();
        if (cudaMemsetAsync(tile_offsets_.get(), 0, (static_cast<size_t>(tile_count) + 1) * sizeof(int64_t), s) !=
            cudaSuccess)
            return false;
    }
    return Blend(cam, background, image);
}

// Per-tile lists by emitting the records in depth order and stable-sorting
// them by tile over all records (record scan, emission, radix sort, ranges).
bool Renderer::OrderBySort(const uint32_t* by_depth, const int* visible, int count, const CameraParams& camera,
                           int tile_count, int64_t* records_out) {
    cudaStream_t s = stream_;
    int* record_count = counters_.get();
    int* overflow = counters_.get() + 1;
    int64_t records = 0;
    gsn::RadixSortScratch scratch;
    bool in_alt = false;
    {
        gsn::stage_mark(s, gsn::kStageRecordScan);
        if (gsn::launch_exclusive_scan(exact_culling_ ? cull_counts_.get() : tile_counts_.get(), by_depth,
                                       record_start_.get(), count, scan_scratch_.get(), s, visible) != GSN_OK)
            return false;
        if (cudaMemcpyAsync(record_count, record_start_.get() + count, sizeof(int), cudaMemcpyDeviceToDevice,
                            s) != cudaSuccess)
            return false;
        if (!fixed_capacity_) {
            if (cudaMemcpyAsync(host_records_, record_count, sizeof(int), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return false;
            records = *host_records_;
            if (records < 0) return false;
            if (!ReserveRecords(records)) return false;
            if (static_cast<size_t>(records) > sort_scratch_count_) {
                size_t want = std::max<size_t>(records, sort_scratch_count_ + sort_scratch_count_ / 2);
                if (!sort_scratch_.Reserve(gsn::radix_sort_scratch_bytes(static_cast<int>(want)))) return false;
                sort_scratch_count_ = want;
            }
            last_records_ = records;
        }
        gsn::stage_mark(s, gsn::kStageEmitRecords);
        const int emitted =
            exact_culling_
                ? gsn::launch_emit_records_culled(by_depth, record_start_.get(), rects_.get(), means_.get(),
                                                  conic_opacities_.get(), count, camera.tile_count_x_,
                                                  tile_keys_[0].get(), record_ids_[0].get(), record_capacity_,
                                                  overflow, s)
                : gsn::launch_emit_records(by_depth, record_start_.get(), rects_.get(), count, camera.tile_count_x_,
                                           tile_keys_[0].get(), record_ids_[0].get(), record_capacity_, overflow,
                                           s);
        if (emitted != GSN_OK) return false;
        const int max_records = fixed_capacity_ ? static_cast<int>(record_capacity_) : static_cast<int>(records);
        scratch = gsn::radix_sort_scratch(sort_scratch_.get(), static_cast<int>(sort_scratch_count_));
        in_alt = false;
        gsn::stage_mark(s, gsn::kStageTileSort);
        if (max_records > 0 &&
            gsn::launch_radix_sort(tile_keys_[0].get(), record_ids_[0].get(), tile_keys_[1].get(),
                                   record_ids_[1].get(), false, max_records,
                                   fixed_capacity_ ? record_count : nullptr, 0, TileBits(tile_count), scratch,
                                   &in_alt, s) != GSN_OK)
            return false;
        sorted_ids_ = record_ids_[in_alt ? 1 : 0].get();
        gsn::stage_mark(s, gsn::kStageTileRanges);
        if (gsn::launch_tile_ranges(tile_keys_[in_alt ? 1 : 0].get(), record_count, std::max(max_records, 1),
                                    tile_count, tile_offsets_.get(), s) != GSN_OK)
            return false;
    }
    *records_out = records;
    return true;
}

// The per-tile blend of the ordered records.
bool Renderer::Blend(const gsn_camera& cam, const float* background, float* image) {
    cudaStream_t s = stream_;
    gsn::RasterForwardArgs ra;
    ra.tile_ids = sorted_ids_;
    ra.tile_offsets = tile_offsets_.get();
    ra.means = means_.get();
    ra.conic_opacity = conic_opacities_.get();
    ra.colors = colors_.get();
    ra.cam = cam;
    ra.background = make_float3(background[0], background[1], background[2]);
    ra.image = image;
    ra.final_transmittance = nullptr;
    ra.contributors = contributors_.get();
    ra.record_warps = record_warps_.get();
    ra.record_words = record_words_;
    ra.fast = fast_blend_;
    ra.pair_count = pair_counter_;
    if (record_warps_.get() &&
        cudaMemsetAsync(record_warps_.get(), 0, 2 * static_cast<size_t>(record_words_) * sizeof(uint32_t), s) !=
            cudaSuccess)
        return false;
    gsn::stage_mark(s, gsn::kStageRasterForward);
    const bool ok = gsn::launch_raster_forward(ra, s) == GSN_OK;
    gsn::stage_mark(s, gsn::kStageOther);
    return ok;
}

const int* Renderer::GetRecordOffsets() const {
    if (!record_offsets_valid_) {
        int n = last_count_;
        if (!record_offsets_.Reserve(static_cast<size_t>(n) + 1)) return nullptr;
        if (!scan_scratch_.get() || static_cast<size_t>(n) > scan_scratch_count_) {
            if (!scan_scratch_.Reserve(gsn::scan_scratch_bytes(std::max(n, 1)))) return nullptr;
            scan_scratch_count_ = static_cast<size_t>(std::max(n, 1));
        }
        if (gsn::launch_exclusive_scan(tile_counts_.get(), nullptr, record_offsets_.get(), n, scan_scratch_.get(),
                                       stream_) != GSN_OK)
            return nullptr;
        record_offsets_valid_ = true;
    }
    return record_offsets_.get();
}

}  // namespace gs_native
