// bvh_build.h — BVH construction on the device (bvh_build.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "flatten.h"

namespace rt {

// Device arrays of a built scene (from the device memory pool of devmem.h;
// the caller returns them).
struct DeviceBvh {
    uint4* nodes = nullptr;      // 8-wide nodes: every BLAS in mesh order, then the TLAS
    float4* tris = nullptr;      // 3 per triangle, BLAS leaf order
    float4* inst_xf = nullptr;   // 3 per instance, scene order
    uint4* inst = nullptr;       // 1 per instance, scene order
    uint2* items = nullptr;      // TLAS primitives (instance, BLAS root child), leaf order
    uint64_t n_nodes = 0;
    std::vector<void*> allocations;
};

// Builds every BLAS and the TLAS of `d` on the device with the host
// builder's rules (flatten.cpp): the same binary trees and byte-identical
// wide nodes; only the order of primitives inside a leaf may differ.
// `H` must come from flatten_scene(d, H, err, false); this fills its mesh
// records (blas_root), tlas_root, world box and node counts. Runs on `st`
// and returns with the stream synchronised. Returns 0 or an RT_ERR_* code
// with `err` set.
int device_build_scene(const rt_scene_desc* d, HostScene* H, DeviceBvh* out, cudaStream_t st, std::string* err);

}  // namespace rt
