// Stage profiler and launch counter (see profile.cpp).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gsn {

enum Stage {
    kStageProject = 0,
    kStageDepthSort,
    kStageRecordScan,
    kStageEmitRecords,
    kStageTileSort,
    kStageTileRanges,
    kStageRasterForward,
    kStageLossGradient,
    kStageRasterBackward,
    kStageGaussianUpdate,
    kStageDensity,
    kStageKnn,
    kStageOther,  // closes the previous stage
    kStageCount
};

void note_launch(int kernels = 1);
uint64_t launch_count();
// Programmatic dependent launch of the training step's kernels (on by default).
void set_programmatic_launch(bool on);
bool programmatic_launch();
void profile_enable(bool on);
bool profile_enabled();
void stage_mark(cudaStream_t stream, int stage);
int profile_collect(double* ms, int count);
const char* stage_name(int stage);

}  // namespace gsn
