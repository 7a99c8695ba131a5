// guide_internal.h — renderer-side access to the learned proposal.
#pragma once

#include <cuda_runtime.h>

#include "guide.cuh"
#include "rt_guide.h"

namespace rt {

// Inference / one training iteration on records whose count lives in device
// memory (*n_dev <= cap), so a render wave needs no host round trip.
// guide_infer_counted returns the raw-output buffer (48 floats per record),
// valid until the next guide call.
int guide_infer_counted(rt_guide* g, const float* rec, const uint32_t* n_dev, uint32_t cap, float** raw_out,
                        cudaStream_t st);
int guide_train_counted(rt_guide* g, const float* rec, const uint32_t* n_dev, uint32_t cap, cudaStream_t st);
const float* guide_loss_ptr(rt_guide* g);
const uint32_t* guide_err_ptr(rt_guide* g);
GuideDev guide_dev(rt_guide* g);

}  // namespace rt
