// em_plan.h -- host-side hooks of the EM engine used by the served form (serve.cu).
#ifndef TGMM_EM_PLAN_H_
#define TGMM_EM_PLAN_H_

#include <cuda_runtime.h>
#include <stddef.h>

#include "../../include/tgmm_gmem.h"

namespace tgmm {

// Bytes of one frame's EM state record.
size_t frame_state_bytes();
// Enqueues on `st` the copy of the per-frame EM state of the batch last launched through
// the plan (n records) into host memory `dst` (pinned, frame_state_bytes() * n).
int plan_enqueue_state(TgmmPlan* P, int32_t n, void* dst, cudaStream_t st);
// Stats of one copied state record; returns the frame's status (TGMM_OK or the code of its
// device flags).
int frame_state_to_stats(const void* state, TgmmEmStats* out);
// Records `what` as the calling thread's last error and returns `code`.
int report_error(int code, const char* what, cudaError_t e);

}  // namespace tgmm

#endif  // TGMM_EM_PLAN_H_
