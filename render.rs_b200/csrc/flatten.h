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
    std::vector<float4> tris1;       // deformation blur: triangles at shutter close (same index), or empty
    std::vector<DevInstMotion> inst_motion;  // transform motion blur: moving instances
    std::vector<uint32_t> inst_mot;  // per instance: its inst_motion entry or ~0 (empty without motion)
    std::vector<float4> inst_xf;     // 3 per instance, scene order
    std::vector<uint4> inst;         // 1 per instance, scene order
    std::vector<uint2> items;        // TLAS primitives, leaf order
    std::vector<MeshInfo> meshes;
    std::vector<uint32_t> orig_idx;
    std::vector<float> normals;
    std::vector<float> st;           // 2 per attribute vertex, empty when no mesh has st
    std::vector<float> inst_scale;   // per instance when the scene has patterns
    std::vector<DevPattern> patterns;
    std::vector<float4> ramp;
    std::vector<DevMatPat> mat_pat;  // per material when the scene has bindings
    std::vector<uint2> binds;
    std::vector<DevPbr> pbr;
    std::vector<DevIes> ies;
    std::vector<float> ies_data;
    std::vector<DevTexture> textures;
    std::vector<DevMip> tex_mips;
    std::vector<float4> texels;
    std::vector<uint2> udim;
    std::vector<DevMaterial> materials;
    std::vector<DevLight> lights;
    std::vector<LightNode> lbvh;
    std::vector<uint32_t> light_leaf;
    std::vector<uint32_t> inf_lights;
    std::vector<float> inf_power;
    std::vector<float4> env;         // environment map texels (RGB, 0)
    std::vector<float> env_marg, env_cond;
    std::vector<DevQuadric> quadrics;
    std::vector<DevMedium> media;
    std::vector<DevHair> hair;
    uint64_t blas_nodes = 0, tlas_nodes = 0, binary_blas_nodes = 0;
    uint64_t n_tris = 0;             // unique triangles over all meshes
    double world_lo[3] = {0, 0, 0}, world_hi[3] = {0, 0, 0};  // union of instance bounds
    double quad_lo[3] = {1e300, 1e300, 1e300}, quad_hi[3] = {-1e300, -1e300, -1e300};  // union of quadric bounds
    DevScene scalars{};              // pointer fields unset; scalar fields filled
};

// Flatten `desc` into device-ready arrays. Returns false with `err` set on
// invalid input (index out of range, non-finite vertex, ...). With
// build_bvh false the BLASes and the TLAS are left to the device builder
// (bvh_build.h): nodes, tris, inst_xf and inst stay empty, mesh records get
// their triangle ranges but no BLAS root, and vertex data is not validated.
bool flatten_scene(const rt_scene_desc* desc, HostScene* out, std::string* err, bool build_bvh = true);

// One child of a mesh's BLAS root: its exact box and its reference (wide
// node index or leaf reference).
struct RootChild {
    float lo[3], hi[3];
    uint32_t ref;
};
// Largest BLAS frontier an instance is split into: a dense scene's
// instances become the second-level frontier (at most 8 x 8 subtrees).
constexpr uint32_t RT_TOP_MAX = 64u;
// The instance-splitting rules of tlas_items (flatten.cpp explains them);
// the device builder's item kernels apply the same.
#ifndef RT_BRAID_RATIO
#define RT_BRAID_RATIO 1.75
#endif
#ifndef RT_BRAID_DENSE
#define RT_BRAID_DENSE 32.0
#endif

// TLAS primitives: every instance contributes one item (instance, BLAS root
// reference) boxed by the union of its root children's world boxes, or one
// item per root child (instance, child reference) when that splits its box
// area well (flatten.cpp: RT_BRAID_RATIO); in a dense scene (instance boxes
// adding up to more than RT_BRAID_DENSE world boxes) one item per node of
// the BLAS's second-level frontier (`grand_children`: each inner root child
// replaced by its children). 6 doubles per item box. Meshes without
// triangles contribute none. Needs H's mesh records (blas_root); sets the
// world box in H. Instance ids must be validated.
void tlas_items(const rt_scene_desc* d, const std::vector<std::vector<RootChild>>& root_children,
                const std::vector<std::vector<RootChild>>& grand_children, std::vector<double>* boxes,
                std::vector<uint2>* items, HostScene* H);

// World-to-object 3x4 of every instance (f32, 3 float4 each, scene order)
// and its record (BLAS root, index, material, mesh).
void instance_records(const rt_scene_desc* d, const HostScene& H, std::vector<float4>* xf, std::vector<uint4>* rec);

// Builder primitive records (8 floats each: lo xyz, index bits, hi xyz, 0)
// of boxes given as 6 doubles: rounded outward to f32, -0 folded into +0.
void prim_records(const std::vector<double>& boxes, float* out);

// f32 material constants as the shade kernel reads them.
DevMaterial fold_material_public(const rt_material_desc& m);
// f32 hair parameters of a hair material.
DevHair hair_dev_public(const rt_material_desc& m);

}  // namespace rt
