/*
 * rt_scene.h — plain-C scene description handed across the C ABI.
 *
 * One descriptor feeds both the CUDA backend (librtcuda.so) and the f64 CPU
 * oracle, so the two always see byte-identical scene input.
 *
 * It replaces the reference's flattened GPU scene payload: `GpuPtScene`
 * (src/raytracer/metal/gpu_scene.rs:254-288) built from `Scene`
 * (src/scene/mod.rs:27-56). Only the parts the path tracer consumes are
 * carried: triangle meshes with optional vertex normals
 * (src/geometry/mesh.rs:20-33), affine instances (mesh.rs:232-250),
 * PxrSurface-lite material parameters (src/scene/pbr.rs:10-51) with emission
 * and the area-light link (src/scene/material.rs:14-40), finite/distant
 * lights (src/scene/light.rs:7-35) and the camera (src/scene/camera.rs:67-92).
 *
 * Doubles are used for every host-side parameter so the f64 oracle reads the
 * same values the reference would; the CUDA backend converts to f32 (and
 * inverts instance transforms in f64) when it flattens the scene.
 *
 * All arrays are borrowed only for the duration of the create call.
 */
#ifndef RT_SCENE_H
#define RT_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Triangle mesh: f32 xyz positions, u32 index triples, optional normals
 * and texture coordinates.
 * Mirrors `Mesh { positions, indices, normals, st }` (src/geometry/mesh.rs:20-33). */
typedef struct rt_mesh_desc {
    const float*    positions;    /* 3 * n_vertices */
    const uint32_t* indices;      /* 3 * n_triangles */
    const float*    normals;      /* 3 * n_vertices, or NULL (geometric normal) */
    uint32_t        n_vertices;
    uint32_t        n_triangles;
    const float*    st;           /* 2 * n_vertices (s, t), or NULL (st = 0, density 0) */
} rt_mesh_desc;

/* Placed copy of a mesh or a curve set. `object_to_world` is the row-major
 * upper 3x4 of the reference's `Instance::transform` (mesh.rs:237); the
 * bottom row is (0,0,0,1). The inverse is computed by the consumer in f64.
 * mesh_id below n_meshes names a mesh, n_meshes + k the curve set k
 * (`Instance::new_curves`, mesh.rs:256-264). */
typedef struct rt_instance_desc {
    double   object_to_world[12];
    uint32_t mesh_id;
    uint32_t material_id;
} rt_instance_desc;

/* Motion blur: shutter-close endpoints (the reference's
 * `Instance::transform1`, mesh.rs:230-235, `Mesh::positions1`,
 * mesh.rs:29-31). Rays draw a shutter time t in [0, 1) per sample when a
 * scene has any endpoint or camera motion (pt/mod.rs:339-356); a moving
 * instance is placed by the component-wise lerp of its two transforms at t
 * (`Instance::transforms_at`, mesh.rs:295-304), a deforming mesh by the
 * lerp of its two vertex positions (`Mesh::vertex_at`, mesh.rs:96-111). */
typedef struct rt_instance_motion {
    uint32_t instance;            /* index into rt_scene_desc::instances */
    uint32_t reserved;            /* 0 */
    double   object_to_world1[12]; /* row-major upper 3x4 at shutter close */
} rt_instance_motion;

typedef struct rt_mesh_motion {
    uint32_t     mesh;            /* index into rt_scene_desc::meshes */
    uint32_t     reserved;        /* 0 */
    const float* positions1;      /* 3 * n_vertices at shutter close (same topology) */
} rt_mesh_motion;

/* Curve set: `CurveSet` (src/geometry/curves.rs:15-26), rounded-cone
 * segments (a swept sphere whose radius goes linearly from the start's to
 * the end's; equal ends make a point particle a sphere). */
typedef struct rt_curves_desc {
    const float* p0;          /* 4 per segment: start xyz, radius */
    const float* p1;          /* 4 per segment: end xyz, radius */
    const float* v0;          /* curve parameter at the start (0 root, 1 tip) */
    const float* v1;          /* and at the end */
    uint32_t n_segments;
    uint32_t reserved;        /* 0 */
} rt_curves_desc;

/* Material: `PbrParams` fields in scope (src/scene/pbr.rs:10-51) plus
 * `Material::{emission, area_light, id}` (src/scene/material.rs:21-39). */
typedef struct rt_material_desc {
    double  diffuse_gain;
    double  diffuse_color[3];
    double  diffuse_roughness;       /* Oren-Nayar sigma (0 = Lambert) */
    double  specular_face_color[3];  /* Schlick F0; black -> from specular_ior */
    double  specular_edge_color[3];  /* Schlick F90 */
    double  specular_roughness;
    double  specular_ior;
    double  clearcoat_gain;
    double  clearcoat_roughness;
    double  fuzz_gain;
    double  fuzz_color[3];
    double  glass_gain;
    double  glass_ior;
    double  glass_roughness;
    double  refraction_color[3];
    double  glow[3];
    double  presence;                /* stochastic cutout alpha, 1 = solid */
    double  emission[3];             /* emitted radiance */
    int32_t area_light;              /* index into lights, or -1 */
    uint32_t id;                     /* object id for the id AOV */
    /* Subsurface random walk (PbrParams::subsurface_*, pbr.rs:43-47):
     * probability of entering the walk, surface colour, mean free path. */
    double  subsurface_gain;
    double  subsurface_color[3];
    double  subsurface_dmfp[3];
    int32_t interior;                /* medium inside this geometry (Material::interior), or -1 */
    uint32_t hair;                   /* 1: Marschner hair on curve hits (Material::hair, pt/hair.rs) */
    double  hair_sigma_a[3];         /* HairParams::sigma_a, absorption per fiber diameter */
    double  hair_beta_m;             /* longitudinal roughness (clamped to [0.01, 1]) */
    double  hair_beta_n;             /* azimuthal roughness (clamped to [0.01, 1]) */
    double  hair_eta;                /* fiber index of refraction */
} rt_material_desc;

enum {
    RT_LIGHT_POINT   = 0,  /* p = position */
    RT_LIGHT_DISTANT = 1,  /* e1 = direction light travels; radius = angular radius */
    RT_LIGHT_RECT    = 2,  /* p = corner, e1/e2 = edges */
    RT_LIGHT_SPHERE  = 3,  /* p = centre, radius */
    RT_LIGHT_DISK    = 4,  /* p = centre, e1/e2 span the radius */
    RT_LIGHT_DOME    = 5   /* constant environment: radiance color * intensity from every direction */
};

/* Light: `Light { light_type, intensity, color }` (src/scene/light.rs:7-49).
 * Radiance is color * intensity (light.rs:151-153). */
typedef struct rt_light_desc {
    int32_t type;
    int32_t pad_;
    double  intensity;
    double  color[3];
    double  p[3];
    double  e1[3];
    double  e2[3];
    double  radius;
} rt_light_desc;

enum { RT_FILTER_BOX = 0, RT_FILTER_TRIANGLE = 1, RT_FILTER_GAUSSIAN = 2 };
/* Camera::projection (camera.rs:5-9). */
enum { RT_PROJECTION_PERSPECTIVE = 0, RT_PROJECTION_ORTHOGRAPHIC = 1 };

/* Pinhole / thin-lens or orthographic camera (src/scene/camera.rs:67-92,
 * 150-179).
 * right/up/forward are used as given (Camera::set_transform computes
 * right = forward x up, up = right x forward). */
typedef struct rt_camera_desc {
    uint32_t width;
    uint32_t height;
    double   fov_deg;               /* vertical field of view */
    double   eye[3];
    double   forward[3];
    double   up[3];
    double   right[3];
    double   lens_radius;           /* 0 = pinhole */
    double   focal_distance;
    int32_t  filter;                /* RT_FILTER_* */
    int32_t  projection;            /* RT_PROJECTION_*; orthographic rays start on the screen window */
    double   filter_width;
    double   ortho_half[2];         /* half-extents of the orthographic window (Camera::ortho_half;
                                       the reference's default is (aspect, 1)) */
} rt_camera_desc;

/* Pattern node (src/texture/pattern.rs:47-67; PatternNode). Every node
 * outputs RGB; scalar consumers read channel 0. */
enum {
    RT_PATTERN_CHECKER       = 0,  /* color_a / color_b cells over st * scale, footprint-filtered */
    RT_PATTERN_FRACTAL       = 1,  /* fBm of classic Perlin noise over world P, remapped to [0,1] */
    RT_PATTERN_MIX           = 2,  /* lerp(in[0], in[1], in[2].r) */
    RT_PATTERN_COLOR_CORRECT = 3,  /* (in[0] * color_a + color_b) ^ (1 / gamma), then saturation */
    RT_PATTERN_RAMP          = 4,  /* piecewise-linear ramp over s (or t) */
    RT_PATTERN_TEXTURE       = 5,  /* file texture over st * scale (trilinear, or EWA along the footprint) */
    RT_PATTERN_TRIPLANAR     = 6   /* file texture projected on the three axis planes of P * frequency */
};

/* Texture wrap modes (src/texture/cache.rs:19-34). */
enum { RT_WRAP_PERIODIC = 0, RT_WRAP_CLAMP = 1, RT_WRAP_BLACK = 2 };

/* A file texture's base image, linear RGB f32, row-major from the top row
 * (what the reference's texture cache holds after txmake,
 * src/texture/tex.rs:71-87); the consumer builds the mip chain. */
typedef struct rt_texture_desc {
    const float* rgb;     /* 3 * width * height */
    uint32_t width;
    uint32_t height;
} rt_texture_desc;

/* Node input (PInput): another node's output or a constant. A node may only
 * read nodes of lower index (the graph is a DAG in index order). */
typedef struct rt_pattern_input {
    int32_t node;       /* index of the node read, or -1 for `value` */
    int32_t pad_;
    double  value[3];
} rt_pattern_input;

typedef struct rt_pattern_desc {
    int32_t  type;                /* RT_PATTERN_* */
    uint32_t octaves;             /* fractal */
    double   color_a[3];          /* checker colour A; colour-correct gain */
    double   color_b[3];          /* checker colour B; colour-correct offset */
    double   scale[2];            /* checker, texture s, t scale */
    double   frequency, gain, lacunarity;  /* fractal; triplanar frequency */
    double   gamma, saturation;   /* colour correct */
    rt_pattern_input in[3];       /* mix: color1, color2, mix; colour correct: in[0] */
    const double* ramp_positions; /* n_ramp, ascending */
    const double* ramp_colors;    /* 3 * n_ramp */
    uint32_t n_ramp;
    uint32_t use_t;               /* ramp over t instead of s */
    int32_t  texture;             /* texture, triplanar: index into textures, -1 = missing (magenta) */
    uint32_t wrap;                /* RT_WRAP_* */
    /* A UDIM tile set instead of one texture (TextureRef::Udim,
     * pattern.rs:14-38): tile numbers 1001 + s cell + 10 t cell and the
     * texture of each; a tile not in the set reads magenta. */
    const uint32_t* udim_tiles;
    const int32_t*  udim_textures;
    uint32_t n_udim;
    uint32_t udim_reserved;       /* 0 */
} rt_pattern_desc;

/* PbrParams fields a pattern output drives (BoundField, pattern.rs:238-254). */
enum {
    RT_FIELD_DIFFUSE_COLOR = 0, RT_FIELD_DIFFUSE_GAIN = 1, RT_FIELD_DIFFUSE_ROUGHNESS = 2,
    RT_FIELD_SPECULAR_FACE_COLOR = 3, RT_FIELD_SPECULAR_EDGE_COLOR = 4, RT_FIELD_SPECULAR_ROUGHNESS = 5,
    RT_FIELD_CLEARCOAT_GAIN = 6, RT_FIELD_FUZZ_GAIN = 7, RT_FIELD_FUZZ_COLOR = 8, RT_FIELD_GLASS_GAIN = 9,
    RT_FIELD_GLASS_ROUGHNESS = 10, RT_FIELD_REFRACTION_COLOR = 11, RT_FIELD_GLOW = 12, RT_FIELD_PRESENCE = 13
};

/* Material::pattern_bindings entry (src/scene/material.rs:29-30): the
 * output of `node` replaces `field` of `material` at every shading point,
 * in binding order. */
typedef struct rt_pattern_binding {
    uint32_t material;
    uint32_t field;     /* RT_FIELD_* */
    uint32_t node;
    uint32_t pad_;
} rt_pattern_binding;

/* IES profile of a point light (src/scene/ies.rs, src/scene/light.rs:
 * 44-45, 155-167): the LM-63 candela grid, already scaled by the file's
 * candela multiplier, over ascending vertical angles (0 = the light's
 * local -y) and horizontal angles, and the rotation taking world
 * directions to the light's frame (the upper 3x3 of the inverse of the
 * light's transform at declaration, row-major). The profile reshapes the
 * light's output, normalised by its sin-weighted mean candela. */
typedef struct rt_ies_desc {
    uint32_t light;            /* index of the RT_LIGHT_POINT light */
    uint32_t n_v;
    uint32_t n_h;
    uint32_t pad_;
    const double* v_angles;    /* n_v, degrees */
    const double* h_angles;    /* n_h, degrees */
    const double* candela;     /* n_h x n_v, candela[h * n_v + v] */
    double world_to_local[9];
} rt_ies_desc;

/* Analytic RiSpec quadrics, the reference's legacy primitives
 * (src/geometry/sphere.rs, cylinder.rs, cone.rs, extra.rs): each is
 * intersected in its own object space (the ray transformed by the inverse
 * of object_to_world, its direction normalised there), its hit distance is
 * the world distance from the ray origin, and the scene tests them all
 * before the meshes, as Scene::intersect's scan of `objects` does
 * (src/scene/mod.rs:105-146). params by type (angles in degrees):
 *   SPHERE       radius, zmin, zmax, thetamax
 *   CYLINDER     radius, zmin, zmax, thetamax
 *   CONE         height, radius, thetamax
 *   TORUS        major radius, minor radius, phimin, phimax, thetamax
 *   DISK         height, radius, thetamax
 *   PARABOLOID   rmax, zmin, zmax, thetamax
 *   HYPERBOLOID  p1 (x, y, z), p2 (x, y, z), thetamax */
enum {
    RT_QUADRIC_SPHERE = 0,
    RT_QUADRIC_CYLINDER = 1,
    RT_QUADRIC_CONE = 2,
    RT_QUADRIC_TORUS = 3,
    RT_QUADRIC_DISK = 4,
    RT_QUADRIC_PARABOLOID = 5,
    RT_QUADRIC_HYPERBOLOID = 6
};
/* Ray-batch results name a quadric hit by this bit in the instance id, the
 * quadric's index in the low bits (its primitive id is 0). */
#define RT_HIT_QUADRIC 0x80000000u

typedef struct rt_quadric_desc {
    double   object_to_world[12];  /* row-major 3x4 */
    double   params[8];
    uint32_t type;                 /* RT_QUADRIC_* */
    uint32_t material_id;
} rt_quadric_desc;

/* Participating medium: `Medium` (src/scene/medium.rs:28-43). Homogeneous
 * when density is RT_DENSITY_NONE; RT_DENSITY_FBM scales the coefficients
 * by clamp((fbm(p) * 0.5 + 0.5 - (1 - coverage)) * sharpness, 0, 1)
 * (medium.rs:56-65, fBm of src/geometry/displace.rs:82-97 with amplitude 1
 * and offset 0). */
enum { RT_DENSITY_NONE = 0, RT_DENSITY_FBM = 1 };
typedef struct rt_medium_desc {
    double   sigma_a[3];
    double   sigma_s[3];
    double   g;               /* Henyey-Greenstein anisotropy */
    double   emission[3];
    double   max_distance;    /* extent along any ray (atmospheres are slabs) */
    uint32_t density;         /* RT_DENSITY_* */
    uint32_t octaves;
    double   frequency, gain, lacunarity, coverage, sharpness;
} rt_medium_desc;

typedef struct rt_scene_desc {
    const rt_mesh_desc*     meshes;
    const rt_instance_desc* instances;
    const rt_material_desc* materials;
    const rt_light_desc*    lights;
    uint32_t n_meshes;
    uint32_t n_instances;
    uint32_t n_materials;
    uint32_t n_lights;
    rt_camera_desc camera;
    double background[3];
    /* Environment map of one dome light (src/scene/envmap.rs): lat-long,
     * env_width x env_height RGB f32 texels, row-major, row 0 at the zenith
     * (+y), column u = atan2(x, -z) / 2pi; NULL for none. */
    const float* env_rgb;
    uint32_t env_width;
    uint32_t env_height;
    uint32_t env_light;       /* index of the RT_LIGHT_DOME light it belongs to */
    uint32_t env_reserved;    /* 0 */
    /* Pattern graph shared by all materials (Scene::patterns,
     * src/scene/mod.rs:39-40) and the material bindings into it. */
    const rt_pattern_desc*    patterns;
    const rt_pattern_binding* bindings;
    uint32_t n_patterns;
    uint32_t n_bindings;
    const rt_texture_desc*    textures;
    uint32_t n_textures;
    uint32_t tex_reserved;    /* 0 */
    const rt_ies_desc*        ies;
    uint32_t n_ies;
    uint32_t ies_reserved;    /* 0 */
    const rt_quadric_desc*    quadrics;
    uint32_t n_quadrics;
    uint32_t quadric_reserved; /* 0 */
    /* Participating media (Scene::media) and the global one (Scene::atmosphere,
     * -1 for none); materials name theirs by rt_material_desc::interior. */
    const rt_medium_desc*     media;
    uint32_t n_media;
    int32_t  atmosphere;
    /* Curve sets (Scene::curve_sets), placed by instances (mesh_id >= n_meshes). */
    const rt_curves_desc*     curves;
    uint32_t n_curves;
    uint32_t curves_reserved; /* 0 */
    /* Motion blur (all NULL / 0 in a static scene): moving instances,
     * deforming meshes (each named at most once), and camera motion, the
     * row-major upper 3x4 of `Camera::motion_inv` (camera.rs:85-146): camera
     * rays at time t are transformed by lerp(I, camera_motion_inv, t), their
     * direction renormalised. Analytic quadrics do not move. */
    const rt_instance_motion* instance_motion;
    uint32_t n_instance_motion;
    uint32_t n_mesh_motion;
    const rt_mesh_motion*     mesh_motion;
    const double*             camera_motion_inv;
} rt_scene_desc;

/* Integrator knobs. The reference hard-codes these as constants
 * (src/raytracer/pt/mod.rs:26-32: MAX_BOUNCES 10, RR_START 3,
 * FIREFLY_CLAMP 60); the configs here need 8/12/16/10 bounces. */
typedef struct rt_params {
    uint32_t max_depth;       /* bounce cap (reference MAX_BOUNCES) */
    uint32_t rr_start;        /* Russian roulette from this depth (RR_START) */
    double   firefly_clamp;   /* per-sample luminance clamp (FIREFLY_CLAMP) */
    uint32_t aovs;            /* 1 = also accumulate the 12-float AOV record */
    uint32_t guided;          /* 1 = learned directional proposal on */
    double   guide_fraction;  /* one-sample MIS fraction drawn from the guide */
    uint64_t max_paths;       /* wavefront slab capacity in paths (0 = auto) */
    double   guide_lr;        /* Adam learning rate of the proposal (0 = 1e-2) */
    uint32_t guide_steps;     /* Adam steps per sample pass when guided (0 = 3) */
    uint32_t guide_depth;     /* guide only vertices of depth < this (0 = all) */
    uint32_t bvh_build;       /* 0 = build the BVHs on the GPU, 1 = on the host (same trees) */
    uint32_t guide_train_passes; /* train the proposal during the first this many sample passes,
                                    then keep it fixed (0 = 512; 0xFFFFFFFF = never stop) */
    uint32_t max_trav_steps;  /* traversal steps one ray may take before the kernel gives it up
                                 and reports RT_ERR_DEVICE (0 = 2^22) */
    uint32_t wait_polls;      /* polls of a tensor-core pipeline wait in the learned proposal's
                                 kernels before they report RT_ERR_DEVICE (0 = 2^24) */
} rt_params;

/* Size checks shared by every consumer of the descriptor. */
#ifdef __cplusplus
static_assert(sizeof(rt_mesh_desc) == 40, "rt_mesh_desc layout");
static_assert(sizeof(rt_instance_desc) == 104, "rt_instance_desc layout");
static_assert(sizeof(rt_material_desc) == 376, "rt_material_desc layout");
static_assert(sizeof(rt_curves_desc) == 40, "rt_curves_desc layout");
static_assert(sizeof(rt_instance_motion) == 104, "rt_instance_motion layout");
static_assert(sizeof(rt_mesh_motion) == 16, "rt_mesh_motion layout");
static_assert(sizeof(rt_medium_desc) == 136, "rt_medium_desc layout");
static_assert(sizeof(rt_light_desc) == 120, "rt_light_desc layout");
static_assert(sizeof(rt_camera_desc) == 160, "rt_camera_desc layout");
static_assert(sizeof(rt_params) == 72, "rt_params layout");
static_assert(sizeof(rt_pattern_input) == 32, "rt_pattern_input layout");
static_assert(sizeof(rt_pattern_desc) == 264, "rt_pattern_desc layout");
static_assert(sizeof(rt_texture_desc) == 16, "rt_texture_desc layout");
static_assert(sizeof(rt_pattern_binding) == 16, "rt_pattern_binding layout");
static_assert(sizeof(rt_ies_desc) == 112, "rt_ies_desc layout");
static_assert(sizeof(rt_quadric_desc) == 168, "rt_quadric_desc layout");
static_assert(sizeof(rt_scene_desc) == 392, "rt_scene_desc layout");
}
#endif

#endif /* RT_SCENE_H */
