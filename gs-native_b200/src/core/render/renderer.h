// Drop-in gs_native::Renderer (reference: src/core/render/renderer.h:10-89).
//
// Same public interface and semantics: Render() projects the 58 x N parameter
// block, builds depth-ordered per-tile record lists and alpha-blends every 16x16
// tile into an fp32 HWC RGB image (`image` is a device pointer, `background` a
// host float[3]). The getters expose the device buffers the Solver consumes.
// Buffers are owned, grow-only and reused across calls; the class is
// non-copyable and not thread-safe, like the reference.
//
// Additions over the reference interface (all optional): an explicit CUDA
// stream, per-pixel contributor counts for the backward pass, the per-Gaussian
// tile counts/rects/depths/radii and a fixed-capacity mode in which Render()
// never waits on the device.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "core/types/buffers.h"
#include "util/device_array.h"

namespace gs_native {

class Renderer {
public:
    Renderer();
    ~Renderer();

    Renderer(const Renderer&) = delete;
    Renderer& operator=(const Renderer&) = delete;

    bool Render(const GaussianBuffers& gaussians, const CameraParams& camera, const float* background,
                float* image, int sh_degree);

    const float2* GetMeans() const { return means_.get(); }
    const float4* GetConicOpacities() const { return conic_opacities_.get(); }
    const float3* GetColors() const { return colors_.get(); }
    const int* GetTileGaussianIds() const { return reinterpret_cast<const int*>(sorted_ids_); }
    const int64_t* GetTileGaussianOffsets() const { return tile_offsets_.get(); }
    // Exclusive scan of the per-Gaussian tile counts in id order (N + 1 entries),
    // computed on first request after each Render().
    const int* GetRecordOffsets() const;
    int GetGaussianCapacity() const { return static_cast<int>(gaussian_capacity_); }
    int GetTileCapacity() const { return static_cast<int>(tile_capacity_); }

    // ---- extensions
    void SetStream(cudaStream_t stream) { stream_ = stream; }
    cudaStream_t GetStream() const { return stream_; }
    // Fixed record capacity: Render() no longer reads the record count back; a
    // frame whose records exceed the capacity sets the overflow flag instead.
    // 0 restores the default grow-on-demand mode.
    bool SetRecordCapacity(int64_t records);
    // Batched form: projection reads the camera from this device pointer (the
    // step frame) instead of the host camera; the host camera still fixes the
    // resolution and tile grid. nullptr restores the host camera.
    void SetDeviceCamera(const gsn_camera* camera) { device_camera_ = camera; }
    // Precision form: the parameter block holds 10 fp32 geometry rows followed
    // by the 48 SH rows in bf16 (34 float rows of stride N).
    void SetBf16Sh(bool enabled) { bf16_sh_ = enabled; }
    // Exact tile culling: emit only the records whose tile the widened
    // alpha >= 1/255 ellipse reaches (the reference emits the whole 3-sigma
    // rectangle). Images and gradients are unchanged; the tile lists are the
    // reference's lists minus records that never contribute. GetTileCounts and
    // GetRecordOffsets keep the rectangle counts (the visibility statistic).
    void SetExactCulling(bool enabled) { exact_culling_ = enabled; }
    // Fast blend arithmetic: the Gaussian power in Horner form with per-record
    // terms hoisted and the hardware exp2 approximation, instead of the
    // reference's per-pixel expression and expf. Images move by a few ulps
    // (no longer bit-identical to the reference); the solver's backward
    // follows the renderer's setting. The fast form also orders depths on
    // 24-bit keys (three radix passes instead of four).
    void SetFastBlend(bool enabled) { fast_blend_ = enabled; }
    bool GetFastBlend() const { return fast_blend_; }
    // Measurement: while set, every Render adds the number of (pixel, record)
    // pairs its blend took to this device counter (a counting variant of the
    // blend kernel; nullptr, the default, runs the plain one).
    void SetPairCounter(unsigned long long* device_counter) { pair_counter_ = device_counter; }
    bool GetExactCulling() const { return exact_culling_; }
    bool GetBf16Sh() const { return bf16_sh_; }
    const int* GetTileCounts() const { return tile_counts_.get(); }
    const int4* GetTileRects() const { return rects_.get(); }
    const float* GetDepths() const { return depths_.get(); }
    const float* GetRadii() const { return radii_.get(); }
    const int* GetContributors() const { return contributors_.get(); }
    // Two bit planes over the records of the last frame (plane w at
    // GetRecordWarps() + w * GetRecordWords()): bit r of plane w is set when a
    // pixel of warp strip w (rows 8w..8w+7 of its tile) took record r in the
    // forward pass. The backward pass skips the others.
    const uint32_t* GetRecordWarps() const { return record_warps_.get(); }
    int64_t GetRecordWords() const { return record_words_; }
    const int* GetRecordCountDevice() const { return counters_.get(); }
    const int* GetOverflowFlag() const { return counters_.get() + 1; }
    int64_t GetRecordCapacity() const { return record_capacity_; }
    // Record count of the last Render() (valid in grow mode without a sync).
    int64_t GetLastRecordCount() const { return last_records_; }
    int GetLastGaussianCount() const { return last_count_; }

private:
    bool ReserveGaussians(int count);
    bool ReserveRecords(int64_t records);

    cudaStream_t stream_ = nullptr;
    size_t gaussian_capacity_ = 0;
    size_t tile_capacity_ = 0;
    int64_t record_capacity_ = 0;
    bool OrderBySort(const uint32_t* by_depth, const int* visible, int count, const CameraParams& camera,
                     int tile_count, int64_t* records_out);
    bool Blend(const gsn_camera& cam, const float* background, float* image);

    bool fixed_capacity_ = false;
    const gsn_camera* device_camera_ = nullptr;
    bool bf16_sh_ = false;
    bool exact_culling_ = false;
    bool fast_blend_ = false;
    unsigned long long* pair_counter_ = nullptr;
    int64_t last_records_ = 0;
    int last_count_ = 0;

    DeviceArray<float2> means_;
    DeviceArray<float4> conic_opacities_;
    DeviceArray<float3> colors_;
    DeviceArray<float> depths_;
    DeviceArray<float> radii_;
    DeviceArray<int4> rects_;
    DeviceArray<int> tile_counts_;
    DeviceArray<int> cull_counts_;  // exact-culling record counts per Gaussian
    DeviceArray<uint32_t> depth_keys_[2];
    DeviceArray<uint32_t> depth_ids_[2];
    DeviceArray<int> record_start_;
    mutable DeviceArray<int> record_offsets_;
    mutable bool record_offsets_valid_ = false;
    DeviceArray<int64_t> tile_offsets_;
    DeviceArray<uint32_t> tile_keys_[2];
    DeviceArray<uint32_t> record_ids_[2];
    uint32_t* sorted_ids_ = nullptr;
    DeviceArray<int> contributors_;
    DeviceArray<uint32_t> record_warps_;
    int64_t record_words_ = 0;
    size_t pixel_capacity_ = 0;
    DeviceArray<unsigned char> sort_scratch_;
    size_t sort_scratch_count_ = 0;
    mutable DeviceArray<unsigned char> scan_scratch_;
    mutable size_t scan_scratch_count_ = 0;
    DeviceArray<int> counters_;  // [0] record count, [1] overflow flag, [2] visible Gaussians
    int* host_records_ = nullptr;  // pinned
};

}  // namespace gs_native
