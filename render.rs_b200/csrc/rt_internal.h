// rt_internal.h — device data layouts shared by the host flattener
// and device BVH builders (flatten.cpp, bvh_build.cu) and the CUDA kernels
// (pt_kernels.cuh, traverse.cuh, shade.cuh).
//
// HBM layout (all arrays 16-byte aligned, read with 128-bit loads):
//   nodes   : 8-wide BVH nodes, 96 B = 6 x uint4 each. Every BLAS (in mesh
//             order) and then the TLAS share one array.
//   tris    : 3 x float4 per triangle in BLAS leaf order, meshes concatenated.
//             (v0.xyz, orig tri id bits) (v1.xyz, -) (v2.xyz, -).
//   items   : uint2 per TLAS primitive in TLAS leaf order: (instance,
//             reference to one child of the instance's BLAS root). The TLAS
//             is built over these instance subtrees (their world boxes are
//             tighter than whole-instance boxes), so a ray enters only the
//             parts of an instance its path crosses.
//   inst_xf : 3 x float4 per instance (scene order): world->object 3x4.
//   inst    : uint4 per instance: (blas root node, original instance id,
//             material id, mesh id).
// The reference's equivalents are 32-B binary nodes, u32 index triples into
// a vertex soup and 224-B instance records (src/raytracer/metal/gpu_scene.rs:
// 20-28, 107-121); the wide layout reads ~3x fewer node bytes per ray.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define RT_HD __host__ __device__
#else
#define RT_HD
#include <vector_types.h>
#include <vector_functions.h>
#endif

namespace rt {

// ---- 8-wide quantised BVH node --------------------------------------------
// word layout (uint4 q[6]):
//   q[0] = (px, py, pz as float bits, ex | ey<<8 | ez<<16 | nchild<<24)
//          child box lo/hi along an axis = p + qbyte * 2^(e-127), exact in f32.
//   q[1] = lo_x[0..7] (bytes), lo_y[0..7]
//   q[2] = lo_z[0..7],         hi_x[0..7]
//   q[3] = hi_y[0..7],         hi_z[0..7]
//   q[4] = ref[0..3], q[5] = ref[4..7]
// ref: 0xFFFFFFFF = empty slot; bit 31 clear = interior child node index;
//      bit 31 set = leaf: bits 0..26 first primitive, bits 27..30 count-1.
static const uint32_t REF_EMPTY = 0xFFFFFFFFu;
static const uint32_t REF_LEAF = 0x80000000u;
static const uint32_t LEAF_FIRST_MASK = (1u << 27) - 1u;
static const int WIDE_NODE_WORDS = 6;

RT_HD inline uint32_t make_leaf_ref(uint32_t first, uint32_t count) {
    return REF_LEAF | ((count - 1u) << 27) | first;
}

// ---- materials (f32, precomputed from PbrParams) -----------------------------
// Lobe weights as PbrParams::lobe_weights (src/scene/pbr.rs:188-201);
// per-lobe constants folded as bxdf.rs evaluates them.
enum MatClass : uint32_t { MAT_DIFFUSE = 0, MAT_CONDUCTOR = 1, MAT_GLASS = 2, MAT_MIXED = 3, MAT_EMITTER = 4 };
static const int N_MAT_CLASSES = 5;

struct DevMaterial {
    float w_diff, w_spec, w_coat, w_fuzz;   // normalised lobe weights
    float w_glass, on_a, on_b, alpha_spec;   // Oren-Nayar A, B; GGX alpha
    float kd[3], alpha_coat;                 // diffuse_color*gain*under_layer/pi
    float f0[3], coat_gain;                  // specular F0
    float f90[3], alpha_glass;               // specular F90 (edge colour)
    float kfuzz[3], glass_scale;             // fuzz_color*gain/pi; glass_gain*under_layer
    float refr[3], ior;                      // refraction colour; glass IOR
    float emission[3], presence;             // emission + glow
    float albedo[3], has_lobes;              // first-hit albedo AOV; 1 if lobes exist
    int32_t area_light;
    uint32_t id;
    uint32_t mclass;
    uint32_t pad_;
};
static_assert(sizeof(DevMaterial) == 160, "DevMaterial layout");

// ---- lights -----------------------------------------------------------------
struct DevLight {
    uint32_t type;
    float radiance[3];    // color * intensity
    float p[3], area;     // point/centre/corner; rect/disk area
    float e1[3], radius;  // rect/disk edge 1 or distant direction; sphere radius or distant angle
    float e2[3], cos_max; // rect/disk edge 2; distant cone cos
    float n[3], pad_;     // rect/disk normal
};
static_assert(sizeof(DevLight) == 80, "DevLight layout");

// Light BVH node, byte-identical to the reference's LightBvhNode
// (src/scene/light_sampler.rs:19-31).
struct LightNode {
    float mn[3];
    float power;
    float mx[3];
    uint32_t parent, a, b;
    uint32_t pad[2];
};
static_assert(sizeof(LightNode) == 48, "LightNode layout");

struct MeshInfo {
    uint32_t idx_base;     // first index of this mesh in orig_idx (3 per tri), or ~0 if no normals
    uint32_t n_tris;
    uint32_t blas_root;
    uint32_t tri_base;     // first triangle (leaf order) in tris
};

// ---- everything a kernel needs to read the scene ------------------------------
struct DevScene {
    const uint4* nodes;
    const float4* tris;
    const float4* inst_xf;
    const uint4* inst;
    const uint2* items;          // TLAS primitives (instance, BLAS child ref), leaf order
    const MeshInfo* meshes;
    const uint32_t* orig_idx;    // original index triples (meshes with normals)
    const float* normals;        // per-vertex normals (meshes with normals)
    const DevMaterial* materials;
    const DevLight* lights;
    const LightNode* lbvh;
    const uint32_t* light_leaf;  // leaf node per light (~0 for infinite)
    const uint32_t* inf_lights;  // infinite-group light ids
    const float* inf_power;
    uint32_t tlas_root;
    uint32_t n_instances;
    uint32_t n_lights;
    uint32_t n_lbvh;
    uint32_t n_inf;
    float inf_total;
    float p_infinite;
    uint32_t any_presence;       // some material has presence < 1
    uint32_t dome;               // first dome light (misses see it), ~0 for none
    // Environment map of light env_light (src/scene/envmap.rs): lat-long
    // texels (RGB + pad), row-marginal CDF (env_h + 1), per-row conditional
    // CDFs (env_w + 1 each) over sin-weighted luminance, their total.
    const float4* env;
    const float* env_marg;
    const float* env_cond;
    uint32_t env_w, env_h, env_light;
    float env_total;
    // camera (src/scene/camera.rs:150-179)
    float eye[3], fwd[3], right[3], up[3];
    float half_w, half_h, lens_radius, focal_distance, filter_width;
    uint32_t filter, width, height;
    float background[3];
};

}  // namespace rt
