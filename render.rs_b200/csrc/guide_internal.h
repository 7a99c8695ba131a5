// guide_internal.h — renderer-side access to the learned proposal.
#pragma once

#include <cuda_runtime.h>

#include "guide.cuh"
#include "rt_guide.h"

namespace rt {

// Inference on records whose count lives in device memory (min(*n_dev, cap)
// records), so a render wave needs no host round trip. Returns the buffer of
// decoded mixtures (48 floats per record, guide.cuh), valid until the next
// guide call.
int guide_infer_counted(rt_guide* g, const float* rec, const uint32_t* n_dev, uint32_t cap, float** raw_out,
                        cudaStream_t st);
// `steps` training iterations over the min(*total_dev, steps * cap) records
// of `rec`, split into equal consecutive slices (at most cap records each).
int guide_train_slices(rt_guide* g, const float* rec, const uint32_t* total_dev, uint32_t cap, uint32_t steps,
                       cudaStream_t st);
// Size the inference buffers for n records up front (no allocation mid-render).
int guide_reserve(rt_guide* g, uint32_t n);
const float* guide_loss_ptr(rt_guide* g);
const uint32_t* guide_err_ptr(rt_guide* g);
GuideDev guide_dev(rt_guide* g);
// Polls of a tensor-core pipeline wait before the network's kernels report
// an error (0 = the default of 2^24).
void guide_set_wait_polls(rt_guide* g, uint32_t polls);

}  // namespace rt
