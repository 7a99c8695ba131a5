// flatten.h — host-side scene flattening for the CUDA backend.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "rt_internal.h"
#include "rt_scene.h"

namespace rt {

struct HostScene {
    std::vector<uint4> nodes;        // 8-wide nodes, 6 words each
    std::vector<float4> tris;        // 3 per triangle, leaf order
    std::vector<float4> inst_xf;     // 3 per instance, TLAS leaf order
    std::vector<uint4> inst;         // 1 per instance, TLAS leaf order
    std::vector<MeshInfo> meshes;
    std::vector<uint32_t> orig_idx;
    std::vector<float> normals;
    std::vector<DevMaterial> materials;
    std::vector<DevLight> lights;
    std::vector<LightNode> lbvh;
    std::vector<uint32_t> light_leaf;
    std::vector<uint32_t> inf_lights;
    std::vector<float> inf_power;
    uint64_t blas_nodes = 0, tlas_nodes = 0, binary_blas_nodes = 0;
    double world_lo[3] = {0, 0, 0}, world_hi[3] = {0, 0, 0};  // union of instance bounds
    DevScene scalars{};              // pointer fields unset; scalar fields filled
};

// Flatten `desc` into device-ready arrays. Returns false with `err` set on
// invalid input (index out of range, non-finite vertex, ...).
bool flatten_scene(const rt_scene_desc* desc, HostScene* out, std::string* err);

// f32 material constants as the shade kernel reads them.
DevMaterial fold_material_public(const rt_material_desc& m);

}  // namespace rt
