// devmem.h — device memory of sessions and BVH builds.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace rt {

// Session and build buffers come from one stream-ordered memory pool per
// device that keeps the blocks it is given back (release threshold: never),
// so a session created after another was destroyed reuses that memory
// without the driver mapping and unmapping gigabytes of path state each
// time (cudaMalloc / cudaFree of ~2 GB took from 20 ms to 0.8 s per call on
// a shared B200 node). Memory is usable on `st` in stream order, and on any
// stream once `st` has been synchronised.
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t st);
// Returns a block to the pool after the work queued on `st` so far.
cudaError_t pool_free(void* p, cudaStream_t st);

}  // namespace rt
