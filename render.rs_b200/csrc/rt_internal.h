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
    uint32_t interior;                       // medium inside (Material::interior), ~0 for none
    // Subsurface random walk: probability, and the Burley-fit homogeneous
    // medium (volume.rs sss_medium) as extinction and scattering.
    float sss_gain, sss_st[3];
    float sss_ss[3], hull;                   // hull: 1 when the surface only bounds `interior`
    uint32_t hair;                           // Marschner parameters in DevScene::hair, ~0 for none
    uint32_t pad2_[3];
};
static_assert(sizeof(DevMaterial) == 208, "DevMaterial layout");

// Marschner hair (src/raytracer/pt/hair.rs HairParams): absorption, IOR,
// the longitudinal variances per lobe and the azimuthal logistic scale.
struct DevHair {
    float sigma_a[3], eta;
    float v[4];
    float s, pad_[3];
};
static_assert(sizeof(DevHair) == 48, "DevHair layout");

// ---- participating media (src/scene/medium.rs) ---------------------------------
struct DevMedium {
    float sigma_a[3], g;
    float sigma_s[3], max_distance;
    float emission[3], majorant;             // channel-max extinction
    float frequency, gain, lacunarity, coverage;
    float sharpness;
    uint32_t octaves, density, pad_;         // density: RT_DENSITY_*
};
static_assert(sizeof(DevMedium) == 80, "DevMedium layout");
#define RT_MAX_MEDIA 127u   // medium indices fit the 7-bit entries of a path's medium stack

// ---- lights -----------------------------------------------------------------
struct DevLight {
    uint32_t type;
    float radiance[3];    // color * intensity
    float p[3], area;     // point/centre/corner; rect/disk area
    float e1[3], radius;  // rect/disk edge 1 or distant direction; sphere radius or distant angle
    float e2[3], cos_max; // rect/disk edge 2; distant cone cos
    float n[3];           // rect/disk normal
    uint32_t ies;         // point light: its IES profile in DevScene::ies, ~0 for none
};
static_assert(sizeof(DevLight) == 80, "DevLight layout");

// IES profile of a point light (src/scene/ies.rs): angles and candela
// (f32) in DevScene::ies_data from `off`: n_v vertical angles, n_h
// horizontal angles, then candela[h][v]; the world-to-light rotation.
struct DevIes {
    uint32_t off, n_v, n_h;
    float average;       // sin-weighted mean candela
    float m[9];          // world -> light, row-major
    uint32_t pad_[3];
};
static_assert(sizeof(DevIes) == 64, "DevIes layout");

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

// Vertex attributes a mesh carries (MeshInfo::attrs).
#define MESH_NORMALS 1u
#define MESH_ST 2u
#define MESH_CURVES 4u   // a curve set: its "triangles" are rounded-cone segments

// A curve segment takes a triangle's 3 float4 in `tris`: (p0 xyz, segment
// id bits) (p1 xyz, r0) (r1, v0, v1, RT_SEG_MARK bits). Triangles keep 0 in
// that last word, so a leaf test tells them apart by it.
#define RT_SEG_MARK 0x7FC5E6u

struct MeshInfo {
    uint32_t idx_base;     // first index of this mesh in orig_idx (3 per tri), or ~0 if no attributes
    uint32_t n_tris;
    uint32_t blas_root;
    uint32_t tri_base;     // first triangle (leaf order) in tris
    uint32_t attrs;        // MESH_NORMALS | MESH_ST
    uint32_t pad_[3];
};
static_assert(sizeof(MeshInfo) == 32, "MeshInfo layout");

// ---- patterns (src/texture/pattern.rs) ------------------------------------------
// One node of the shared pattern graph. Inputs are node indices (below the
// node's own) or ~0 for the constant in c[k].
struct DevPattern {
    uint32_t type;           // RT_PATTERN_*
    uint32_t in[3];
    float c[3][3];           // input constants; checker colours A, B in c[0], c[1];
                             // colour-correct gain, offset in c[1], c[2]
    float s0, s1, s2;        // checker s, t scale | fractal frequency, gain, lacunarity |
                             // colour-correct gamma, saturation
    uint32_t u0, u1, u2;     // fractal octaves | ramp first entry, entries, use_t |
                             // texture index (~0 missing), wrap, UDIM tiles (0: one texture)
    uint32_t udim_off;       // UDIM set: first (tile, texture) entry in DevScene::udim
};
static_assert(sizeof(DevPattern) == 80, "DevPattern layout");

// Base PbrParams of a patterned material (f32), re-folded at every hit
// after the pattern outputs are substituted.
struct DevPbr {
    float diffuse_gain, diffuse_color[3], diffuse_roughness;
    float spec_face[3], spec_edge[3], spec_rough, spec_ior;
    float cc_gain, cc_rough;
    float fuzz_gain, fuzz_color[3];
    float glass_gain, glass_ior, glass_rough;
    float refraction[3], glow[3], presence, emission[3];
    float sss_albedo[3], pad_;   // subsurface colour x gain, the first-hit albedo's share
};
static_assert(sizeof(DevPbr) == 144, "DevPbr layout");

// Per material: its bindings (binds[bind_off .. bind_off + bind_n) as
// (field, node)), the nodes they reach (node_lo + bit k of node_mask),
// and its base parameters (pbr[pbr_index]).
struct DevMatPat {
    uint32_t bind_off, bind_n, node_lo, node_mask;
    uint32_t pbr_index, pad_[3];
};
static_assert(sizeof(DevMatPat) == 32, "DevMatPat layout");
#define RT_MAX_PATTERN_NODES 16

// File textures: every mip level of every texture, RGB texels as float4
// (w = 0) row-major from the top row, concatenated in `texels`.
struct DevTexture {
    uint32_t first_mip, n_mips;
    float base;              // max(width, height) of the base level
    uint32_t pad_;
};
struct DevMip {
    uint32_t offset, w, h, pad_;  // first texel in `texels`, size
};
static_assert(sizeof(DevTexture) == 16 && sizeof(DevMip) == 16, "texture table layout");

// ---- everything a kernel needs to read the scene ------------------------------
// Analytic quadric (rt_quadric_desc) in f32: both transforms, the
// parameters, and Matrix4::approx_scale of object_to_world.
struct DevQuadric {
    float4 w2o[3];      // world -> object rows (3x4)
    float4 o2w[3];      // object -> world rows (3x4)
    float prm[8];
    uint32_t type, material;
    float scale, pad_;
};
static_assert(sizeof(DevQuadric) == 144, "DevQuadric layout");
// Closest-hit records name a quadric hit by this bit in the triangle field
// (leaf-order triangle indices stay below it); the low bits are its index.
#define RT_TRI_QUADRIC 0x80000000u

// Transform motion blur (Instance::transform1, src/geometry/mesh.rs:230-304):
// a moving instance's object-to-world rows at shutter open and close (f32);
// a ray at shutter time t > 0 enters it through the inverse of their
// component-wise lerp.
struct DevInstMotion {
    float4 o2w0[3], o2w1[3];
};
static_assert(sizeof(DevInstMotion) == 96, "DevInstMotion layout");
// Deformation blur (Mesh::positions1, mesh.rs:29-31, 96-111): the second
// record of a deforming mesh's triangle carries this mark in w, and the
// scene's second triangle array holds the triangle at shutter close.
#define RT_DEFORM_MARK 0x7FC5E7u

// Ray pump refill thresholds (lanes of a warp still holding a ray when the
// idle ones are refilled). Measured on B200 (one 1280x720 pass of the
// 772k-instance forest, the 1920x1080 cloud at 8 spp): refilling at 20, 26,
// 28, 30, 32 lanes took the forest 173, 164, 162, 163, 171 ms and the cloud
// 50.5, 52.3, 54.3, 58.1, 60.5 ms. The forest's long rays through
// overlapping instances leave lanes idle unevenly, so scenes whose
// instances overlap densely (the TLAS builders' dense rule) refill earlier.
constexpr uint32_t RT_REFILL_SPARSE = 20, RT_REFILL_DENSE = 28;

struct DevScene {
    const uint4* nodes;
    const float4* tris;
    const float4* inst_xf;
    const uint4* inst;
    const uint2* items;          // TLAS primitives (instance, BLAS child ref), leaf order
    const MeshInfo* meshes;
    const uint32_t* orig_idx;    // original index triples (meshes with normals or st)
    const float* normals;        // per-vertex normals (meshes with attributes; 0 without normals)
    const float* st;             // per-vertex (s, t) (same numbering), or null without any st
    const float* inst_scale;     // Matrix4::approx_scale per instance (scene order), or null
    // Pattern graph (null when the scene has none).
    const DevPattern* patterns;
    const float4* ramp;          // (position, r, g, b) ramp entries
    const DevMatPat* mat_pat;    // per material
    const uint2* binds;          // (field, node)
    const DevPbr* pbr;
    const DevIes* ies;           // IES profiles (null when none)
    const float* ies_data;
    const DevTexture* textures;  // file textures (null when none)
    const DevMip* tex_mips;
    const float4* texels;
    const uint2* udim;           // UDIM sets: (tile number, texture index or ~0)
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
    const DevQuadric* quadrics;  // analytic quadrics, tested before the BVH (null when none)
    uint32_t n_quadrics;
    uint32_t any_presence;       // some material has presence < 1
    uint32_t presence_pat;       // some material's presence is bound to a pattern (texture cutouts)
    uint32_t max_steps;          // traversal steps per ray before the query is given up (error bit)
    uint32_t refill_at;          // ray pump: refill idle lanes once at most this many hold a ray
    uint32_t dome;               // first dome light (misses see it), ~0 for none
    const DevMedium* media;      // participating media (null when none)
    uint32_t n_media;
    uint32_t atmosphere;         // global medium, ~0 for none
    uint32_t any_sss;            // some material has a subsurface walk
    const DevHair* hair;         // hair parameters (null when no material has them)
    uint32_t any_curves;         // the scene has curve sets
    // Environment map of light env_light (src/scene/envmap.rs): lat-long
    // texels (RGB + pad), row-marginal CDF (env_h + 1), per-row conditional
    // CDFs (env_w + 1 each) over sin-weighted luminance, their total.
    const float4* env;
    const float* env_marg;
    const float* env_cond;
    uint32_t env_w, env_h, env_light;
    float env_total;
    // Motion blur (null / 0 in a static scene): rays draw a shutter time
    // (pt/mod.rs:339-356); moving instances, by index (inst_mot: ~0 for a
    // static instance); triangles at shutter close (leaf order, entries of
    // static meshes unused); camera motion, the 3x4 rows of
    // Camera::motion_inv (camera.rs:134-146).
    const DevInstMotion* inst_motion;
    const uint32_t* inst_mot;
    const float4* tris1;
    uint32_t motion;
    uint32_t cam_moving;
    float cam_mot[12];
    // camera (src/scene/camera.rs:150-179)
    float eye[3], fwd[3], right[3], up[3];
    float half_w, half_h, lens_radius, focal_distance, filter_width;
    uint32_t filter, width, height;
    uint32_t projection;         // RT_PROJECTION_*
    float ortho_hw, ortho_hh;    // orthographic window half-extents
    float background[3];
};

}  // namespace rt
