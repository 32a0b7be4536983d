// gs_native::MultiViewRenderer over csrc/multiview.cu and the single-view
// ordering kernels of csrc/sort.cu.
#include "core/render/multiview_renderer.h"

#include <algorithm>
#include <climits>
#include <cstring>

#include "kernels.h"
#include "multiview.h"

namespace gs_native {

struct MultiViewRenderer::View {
    DeviceArray<float2> means;
    DeviceArray<float4> conic;
    DeviceArray<float3> colors;
    DeviceArray<float> depths;
    DeviceArray<int4> rects;
    DeviceArray<int> tile_counts;
    DeviceArray<uint32_t> depth_keys[2], depth_ids[2];
    DeviceArray<int> record_start;
    DeviceArray<int64_t> tile_offsets;
    DeviceArray<uint32_t> tile_keys[2], record_ids[2], record_depth;
    DeviceArray<unsigned char> sort_scratch, scan_scratch;
    size_t gaussians = 0;
    int64_t record_capacity = 0;
    size_t tile_capacity = 0;
    size_t sort_scratch_count = 0;
    const uint32_t* by_depth = nullptr;
    const uint32_t* sorted_ids = nullptr;
    gsn_camera cam{};
    int tiles = 0;
    int64_t records = 0;
};

MultiViewRenderer::MultiViewRenderer() = default;

MultiViewRenderer::~MultiViewRenderer() {
    if (host_totals_) cudaFreeHost(host_totals_);
    for (cudaEvent_t e : joins_) cudaEventDestroy(e);
    if (fork_) cudaEventDestroy(fork_);
    for (cudaStream_t st : side_) cudaStreamDestroy(st);
}

bool MultiViewRenderer::EnsureSideStreams() {
    if (!side_.empty()) return true;
    if (cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming) != cudaSuccess) {
        fork_ = nullptr;
        return false;
    }
    for (int k = 0; k < kSideStreams; ++k) {
        cudaStream_t st = nullptr;
        cudaEvent_t e = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return false;
        side_.push_back(st);
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
        joins_.push_back(e);
    }
    return true;
}

bool MultiViewRenderer::ConfigValid(const MultiViewConfig& c) {
    return gsn::multiview_config_valid(c.tile_w, c.tile_h, c.threads) &&
           (c.key_bits == 32 || c.key_bits == 48 || c.key_bits == 64);
}

bool MultiViewRenderer::SetConfig(const MultiViewConfig& config) {
    if (!ConfigValid(config)) return false;
    config_ = config;
    return true;
}

namespace {

int Bits(int tiles) {
    int b = 0;
    for (unsigned int t = static_cast<unsigned int>(std::max(tiles - 1, 0)); t; t >>= 1) ++b;
    return std::max(b, 1);
}

bool SortScratch(DeviceArray<unsigned char>& scratch, size_t& have, int64_t need) {
    if (need <= static_cast<int64_t>(have) && scratch.get()) return true;
    const size_t want = std::max<size_t>(static_cast<size_t>(need), have + have / 2);
    if (want > static_cast<size_t>(INT_MAX)) return false;
    if (!scratch.Reserve(gsn::radix_sort_scratch_bytes(static_cast<int>(want)))) return false;
    have = want;
    return true;
}

}  // namespace

bool MultiViewRenderer::Prepare(View& v, const GaussianBuffers& g, const CameraParams& camera, int sh_degree,
                                cudaStream_t stream) {
    const int n = g.gaussian_count_;
    v.cam = AsGsnCamera(camera);
    v.cam.tile_count_x = (camera.width_ + config_.tile_w - 1) / config_.tile_w;
    v.cam.tile_count_y = (camera.height_ + config_.tile_h - 1) / config_.tile_h;
    v.tiles = v.cam.tile_count_x * v.cam.tile_count_y;
    const size_t N = static_cast<size_t>(std::max(n, 1));
    if (N > v.gaussians) {
        if (!v.means.Reserve(N) || !v.conic.Reserve(N) || !v.colors.Reserve(N) || !v.depths.Reserve(N) ||
            !v.rects.Reserve(N) || !v.tile_counts.Reserve(N) || !v.depth_keys[0].Reserve(N) ||
            !v.depth_keys[1].Reserve(N) || !v.depth_ids[0].Reserve(N) || !v.depth_ids[1].Reserve(N) ||
            !v.record_start.Reserve(N + 1) || !v.scan_scratch.Reserve(gsn::scan_scratch_bytes(static_cast<int>(N))))
            return false;
        v.gaussians = N;
    }
    if (static_cast<size_t>(v.tiles) + 1 > v.tile_capacity) {
        if (!v.tile_offsets.Reserve(static_cast<size_t>(v.tiles) + 1)) return false;
        v.tile_capacity = static_cast<size_t>(v.tiles) + 1;
    }
    if (!SortScratch(v.sort_scratch, v.sort_scratch_count, n)) return false;
    gsn::ProjectOutputs po{v.means.get(), v.conic.get(), v.colors.get(), v.depths.get(),
                           v.rects.get(), v.tile_counts.get(), v.depth_keys[0].get(), nullptr, nullptr, 0};
    if (gsn::launch_project_tiled(g.gaussians_, n, v.cam, config_.tile_w, config_.tile_h, sh_degree, po, stream) !=
        GSN_OK)
        return false;
    if (config_.key_bits == 32) {
        gsn::RadixSortScratch scratch = gsn::radix_sort_scratch(v.sort_scratch.get(), static_cast<int>(v.sort_scratch_count));
        bool alt = false;
        if (gsn::launch_radix_sort(v.depth_keys[0].get(), v.depth_ids[0].get(), v.depth_keys[1].get(),
                                   v.depth_ids[1].get(), true, n, nullptr, 0, 32, scratch, &alt, stream) != GSN_OK)
            return false;
        v.by_depth = v.depth_ids[alt ? 1 : 0].get();
        return gsn::launch_exclusive_scan(v.tile_counts.get(), v.by_depth, v.record_start.get(), n,
                                          v.scan_scratch.get(), stream) == GSN_OK;
    }
    v.by_depth = nullptr;
    return gsn::launch_exclusive_scan(v.tile_counts.get(), nullptr, v.record_start.get(), n, v.scan_scratch.get(),
                                      stream) == GSN_OK;
}

bool MultiViewRenderer::Order(View& v, int n, cudaStream_t stream) {
    const int64_t r = v.records;
    if (r > v.record_capacity) {
        const int64_t grow = std::min<int64_t>(std::max<int64_t>(r, v.record_capacity + v.record_capacity / 2), INT_MAX);
        if (grow < r || !v.tile_keys[0].Reserve(grow) || !v.tile_keys[1].Reserve(grow) ||
            !v.record_ids[0].Reserve(grow) || !v.record_ids[1].Reserve(grow) || !v.record_depth.Reserve(grow))
            return false;
        v.record_capacity = grow;
    }
    if (!SortScratch(v.sort_scratch, v.sort_scratch_count, std::max<int64_t>(r, n))) return false;
    gsn::RadixSortScratch scratch = gsn::radix_sort_scratch(v.sort_scratch.get(), static_cast<int>(v.sort_scratch_count));
    const int records = static_cast<int>(r);
    bool alt = false;
    if (config_.key_bits == 32) {
        if (gsn::launch_emit_records(v.by_depth, v.record_start.get(), v.rects.get(), n, v.cam.tile_count_x,
                                     v.tile_keys[0].get(), v.record_ids[0].get(), v.record_capacity, nullptr,
                                     stream) != GSN_OK)
            return false;
        if (records > 0 &&
            gsn::launch_radix_sort(v.tile_keys[0].get(), v.record_ids[0].get(), v.tile_keys[1].get(),
                                   v.record_ids[1].get(), false, records, nullptr, 0, Bits(v.tiles), scratch, &alt,
                                   stream) != GSN_OK)
            return false;
    } else {
        // records in id order with their depth key; stable sort on depth (the
        // values are record indices), gather, stable sort on the tile key
        if (gsn::launch_emit_keyed(v.record_start.get(), v.rects.get(), v.tile_counts.get(), v.depth_keys[0].get(),
                                   n, v.cam.tile_count_x, v.record_capacity, v.tile_keys[0].get(),
                                   v.record_depth.get(), v.record_ids[0].get(), stream) != GSN_OK)
            return false;
        if (records > 0) {
            bool depth_alt = false;
            // depth keys -> record_depth / tile_keys[1] ping-pong, record order -> record_ids[1] / depth_ids[1]
            uint32_t* keys = v.record_depth.get();
            uint32_t* keys_alt = v.tile_keys[1].get();
            uint32_t* order = v.record_ids[1].get();
            uint32_t* order_alt = v.depth_ids[1].Reserve(static_cast<size_t>(records)) ? v.depth_ids[1].get() : nullptr;
            if (!order_alt ||
                gsn::launch_radix_sort(keys, order, keys_alt, order_alt, true, records, nullptr, 0, 32, scratch,
                                       &depth_alt, stream) != GSN_OK)
                return false;
            const uint32_t* sorted_order = depth_alt ? order_alt : order;
            // gathered (tile, id) pairs into record_depth / tile_keys[1]
            if (gsn::launch_gather_records(sorted_order, v.tile_keys[0].get(), v.record_ids[0].get(), records,
                                           v.record_depth.get(), v.tile_keys[1].get(), stream) != GSN_OK)
                return false;
            const int bits = config_.key_bits == 48 ? Bits(v.tiles) : 32;
            bool tile_alt = false;
            if (gsn::launch_radix_sort(v.record_depth.get(), v.tile_keys[1].get(), v.tile_keys[0].get(),
                                       v.record_ids[0].get(), false, records, nullptr, 0, bits, scratch, &tile_alt,
                                       stream) != GSN_OK)
                return false;
            v.sorted_ids = tile_alt ? v.record_ids[0].get() : v.tile_keys[1].get();
            const uint32_t* sorted_tiles = tile_alt ? v.tile_keys[0].get() : v.record_depth.get();
            return gsn::launch_tile_ranges(sorted_tiles, v.record_start.get() + n, std::max(records, 1), v.tiles,
                                           v.tile_offsets.get(), stream) == GSN_OK;
        }
    }
    v.sorted_ids = v.record_ids[alt ? 1 : 0].get();
    if (records == 0)
        return cudaMemsetAsync(v.tile_offsets.get(), 0, (static_cast<size_t>(v.tiles) + 1) * sizeof(int64_t),
                               stream) == cudaSuccess;
    return gsn::launch_tile_ranges(v.tile_keys[alt ? 1 : 0].get(), v.record_start.get() + n, records, v.tiles,
                                   v.tile_offsets.get(), stream) == GSN_OK;
}

bool MultiViewRenderer::Render(const GaussianBuffers& g, const std::vector<CameraParams>& cameras,
                               const float background[3], const std::vector<float*>& images, int sh_degree) {
    const int n = g.gaussian_count_;
    const size_t count = cameras.size();
    if (count == 0 || images.size() != count || !background || n <= 0 || !g.gaussians_) return false;
    for (size_t k = 0; k < count; ++k)
        if (!images[k] || cameras[k].width_ <= 0 || cameras[k].height_ <= 0) return false;
    while (views_.size() < count) views_.push_back(std::make_unique<View>());
    if (host_totals_count_ < count) {
        if (host_totals_) cudaFreeHost(host_totals_);
        if (cudaMallocHost(&host_totals_, count * sizeof(int)) != cudaSuccess) {
            host_totals_ = nullptr;
            host_totals_count_ = 0;
            return false;
        }
        host_totals_count_ = count;
    }
    sh_degree = std::clamp(sh_degree, 0, 3);
    if (!EnsureSideStreams()) return false;
    // the views' preprocessing runs on side streams, view k on side stream
    // k % kSideStreams, after the work already queued on the caller's stream
    if (cudaEventRecord(fork_, stream_) != cudaSuccess) return false;
    for (cudaStream_t side : side_)
        if (cudaStreamWaitEvent(side, fork_, 0) != cudaSuccess) return false;
    auto side_of = [&](size_t k) { return side_[k % side_.size()]; };
    // phase 1: projection and record counts of every view, one readback
    for (size_t k = 0; k < count; ++k) {
        if (!Prepare(*views_[k], g, cameras[k], sh_degree, side_of(k)) ||
            cudaMemcpyAsync(host_totals_ + k, views_[k]->record_start.get() + n, sizeof(int), cudaMemcpyDeviceToHost,
                            side_of(k)) != cudaSuccess)
            return false;
    }
    for (cudaStream_t side : side_)
        if (cudaStreamSynchronize(side) != cudaSuccess) return false;
    // phase 2: record ordering and ranges of every view, then the caller's
    // stream waits for all of them
    last_records_ = 0;
    for (size_t k = 0; k < count; ++k) {
        if (host_totals_[k] < 0) return false;
        views_[k]->records = host_totals_[k];
        last_records_ += host_totals_[k];
        if (!Order(*views_[k], n, side_of(k))) return false;
    }
    for (size_t j = 0; j < side_.size(); ++j)
        if (cudaEventRecord(joins_[j], side_[j]) != cudaSuccess || cudaStreamWaitEvent(stream_, joins_[j], 0) != cudaSuccess)
            return false;
    // one persistent blend over all (view, tile) work items
    std::vector<gsn::MultiView> table(count);
    std::vector<int> prefix(count + 1, 0);
    for (size_t k = 0; k < count; ++k) {
        const View& v = *views_[k];
        gsn::MultiView& t = table[k];
        t.tile_ids = v.sorted_ids;
        t.tile_offsets = v.tile_offsets.get();
        t.means = v.means.get();
        t.conic_opacity = v.conic.get();
        t.colors = v.colors.get();
        t.image = images[k];
        t.width = v.cam.width;
        t.height = v.cam.height;
        t.tiles_x = v.cam.tile_count_x;
        t.tiles_y = v.cam.tile_count_y;
        t.background = make_float3(background[0], background[1], background[2]);
        prefix[k + 1] = prefix[k] + v.tiles;
    }
    const size_t table_bytes = count * sizeof(gsn::MultiView);
    const size_t prefix_bytes = (count + 1) * sizeof(int);
    const size_t bytes = table_bytes + prefix_bytes + sizeof(int);
    if (!table_.Reserve(bytes)) return false;
    // the table is staged through a host buffer that lives until the copy is done
    std::vector<unsigned char> host(bytes, 0);
    std::memcpy(host.data(), table.data(), table_bytes);
    std::memcpy(host.data() + table_bytes, prefix.data(), prefix_bytes);
    if (cudaMemcpyAsync(table_.get(), host.data(), bytes, cudaMemcpyHostToDevice, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
        return false;
    gsn::MultiViewArgs a{};
    a.views = reinterpret_cast<const gsn::MultiView*>(table_.get());
    a.tile_prefix = reinterpret_cast<const int*>(table_.get() + table_bytes);
    a.queue = reinterpret_cast<int*>(table_.get() + table_bytes + prefix_bytes);
    a.view_count = static_cast<int>(count);
    a.total_tiles = prefix[count];
    return gsn::launch_multiview(a, config_.tile_w, config_.tile_h, config_.threads, stream_) == GSN_OK;
}

bool MultiViewRenderer::Autotune(const GaussianBuffers& g, const std::vector<CameraParams>& cameras,
                                 const float background[3], const std::vector<float*>& images, int sh_degree,
                                 int repeats, std::vector<MultiViewTiming>* timings) {
    repeats = std::max(repeats, 1);
    const MultiViewConfig start = config_;
    std::vector<MultiViewTiming> all;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return false;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return false;
    }
    bool ok = true;
    for (int tw_th : {0, 1, 2}) {
        const int tw = tw_th == 2 ? 8 : 16, th = tw_th == 0 ? 16 : 8;
        for (int threads : {64, 128, 256})
            for (int bits : {32, 48, 64}) {
                MultiViewConfig c{tw, th, threads, bits};
                if (!ConfigValid(c)) continue;
                config_ = c;
                ok = ok && Render(g, cameras, background, images, sh_degree);  // warm-up (allocations)
                ok = ok && cudaEventRecord(e0, stream_) == cudaSuccess;
                for (int r = 0; r < repeats && ok; ++r) ok = Render(g, cameras, background, images, sh_degree);
                ok = ok && cudaEventRecord(e1, stream_) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
                float ms = 0.0f;
                ok = ok && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
                if (!ok) break;
                all.push_back({c, static_cast<double>(ms) / repeats});
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok || all.empty()) {
        config_ = start;
        return false;
    }
    const auto best = std::min_element(all.begin(), all.end(),
                                       [](const MultiViewTiming& a, const MultiViewTiming& b) { return a.ms < b.ms; });
    config_ = best->config;
    if (timings) *timings = all;
    return true;
}

}  // namespace gs_native
