// Step-frame kernel of the batched form: at the start of every captured
// iteration one warp reads the schedule entry of the step and writes the
// view's camera, target pointer, position learning rate and Adam bias
// corrections into the device frame that the projection, loss and update
// kernels of the same graph read. No host work happens between steps.
#include "common.cuh"
#include "kernels.h"

namespace gsn {

namespace {

__global__ void __launch_bounds__(32) advance_frame_kernel(StepSchedule s, StepFrame* __restrict__ f) {
    pdl_begin();
    __shared__ int step, view;
    if (threadIdx.x == 0) {
        // a record overflow of the previous step is folded in before the
        // renderer clears its flag
        if (s.overflow && *s.overflow) atomicExch(s.status, GSN_ERR_CAPACITY);
        int k = *s.cursor;
        if (k >= s.steps) {
            atomicExch(s.status, GSN_ERR_CAPACITY);
            k = s.steps - 1;
        } else {
            *s.cursor = k + 1;
        }
        int v = s.views[k];
        if (v < 0 || v >= s.view_count) {
            atomicExch(s.status, GSN_ERR_CAPACITY);
            v = 0;
        }
        step = k;
        view = v;
    }
    __syncthreads();
    const uint32_t* src = reinterpret_cast<const uint32_t*>(s.cameras + view);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&f->cam);
    for (int w = threadIdx.x; w < static_cast<int>(sizeof(gsn_camera) / 4); w += 32) dst[w] = src[w];
    if (threadIdx.x == 0) {
        f->target = s.targets + view * s.target_stride;
        f->position_lr = s.position_lr[step];
        f->c1 = s.c1[step];
        f->c2 = s.c2[step];
        f->seed = s.seeds[step];
        f->view = view;
        f->step = step;
    }
}

}  // namespace

int launch_advance_frame(const StepSchedule& s, StepFrame* frame, cudaStream_t stream) {
    if (!frame || !s.cameras || !s.targets || !s.views || !s.position_lr || !s.c1 || !s.c2 || !s.seeds || !s.cursor ||
        !s.status || s.steps <= 0 || s.view_count <= 0)
        return GSN_ERR_INVALID_ARGUMENT;
    launch_step(advance_frame_kernel, 1, 32, 0, stream, s, frame);
    return launched(1);
}

}  // namespace gsn
