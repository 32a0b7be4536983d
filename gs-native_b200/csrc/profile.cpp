// Stage profiler and launch counter of the gs-native library.
//
// When enabled, every stage boundary records a CUDA event on the stream the
// stage runs on; Collect() turns consecutive events into per-stage device time.
// Disabled (the default) it costs one relaxed atomic load per stage boundary.
// Every kernel launch site bumps a process-wide launch counter, which the
// benchmark reports as the number of this library's kernels in its timed region.
#include "profile.h"

#include <atomic>
#include <mutex>
#include <vector>

namespace gsn {

namespace {

std::atomic<uint64_t> g_launches{0};
std::atomic<bool> g_enabled{false};

struct Mark {
    int stage;
    cudaEvent_t event;
    cudaStream_t stream;
};

std::mutex g_mutex;
std::vector<Mark> g_marks;
std::vector<cudaEvent_t> g_pool;

const char* kNames[kStageCount] = {"project",       "depth_sort",     "record_scan",     "emit_records",
                                   "tile_sort",     "tile_ranges",    "raster_forward",  "loss_gradient",
                                   "raster_backward", "gaussian_update", "density",       "knn",
                                   "other"};

}  // namespace

void note_launch(int kernels) { g_launches.fetch_add(static_cast<uint64_t>(kernels), std::memory_order_relaxed); }

namespace {
std::atomic<bool> g_programmatic_launch{true};
}  // namespace

void set_programmatic_launch(bool on) { g_programmatic_launch.store(on, std::memory_order_relaxed); }
bool programmatic_launch() { return g_programmatic_launch.load(std::memory_order_relaxed); }

uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

void profile_enable(bool on) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_enabled.store(on);
    g_marks.clear();
}

bool profile_enabled() { return g_enabled.load(std::memory_order_relaxed); }

void stage_mark(cudaStream_t stream, int stage) {
    if (!g_enabled.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lock(g_mutex);
    cudaEvent_t e;
    if (!g_pool.empty()) {
        e = g_pool.back();
        g_pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
        return;
    }
    cudaEventRecord(e, stream);
    g_marks.push_back({stage, e, stream});
}

int profile_collect(double* ms, int count) {
    std::lock_guard<std::mutex> lock(g_mutex);
    for (int k = 0; k < count && k < kStageCount; ++k) ms[k] = 0.0;
    if (g_marks.empty()) return 0;
    if (cudaEventSynchronize(g_marks.back().event) != cudaSuccess) return -1;
    for (size_t i = 0; i + 1 < g_marks.size(); ++i) {
        const Mark& a = g_marks[i];
        const Mark& b = g_marks[i + 1];
        if (a.stage < 0 || a.stage >= count || a.stream != b.stream) continue;
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, a.event, b.event) == cudaSuccess) ms[a.stage] += t;
    }
    for (const Mark& m : g_marks) g_pool.push_back(m.event);
    g_marks.clear();
    return 0;
}

const char* stage_name(int stage) { return stage >= 0 && stage < kStageCount ? kNames[stage] : "?"; }

}  // namespace gsn
