"""ctypes mirrors of ``include/rt_scene.h`` and ``include/rt_cuda.h``.

The field order and sizes are asserted against the C headers' static
assertions so a drift between the two fails at import time.
"""
import ctypes as C

c_double3 = C.c_double * 3


class RtMeshDesc(C.Structure):
    _fields_ = [
        ("positions", C.POINTER(C.c_float)),
        ("indices", C.POINTER(C.c_uint32)),
        ("normals", C.POINTER(C.c_float)),
        ("n_vertices", C.c_uint32),
        ("n_triangles", C.c_uint32),
        ("st", C.POINTER(C.c_float)),
    ]


class RtInstanceDesc(C.Structure):
    _fields_ = [
        ("object_to_world", C.c_double * 12),
        ("mesh_id", C.c_uint32),
        ("material_id", C.c_uint32),
    ]


class RtInstanceMotion(C.Structure):
    _fields_ = [
        ("instance", C.c_uint32),
        ("reserved", C.c_uint32),
        ("object_to_world1", C.c_double * 12),
    ]


class RtMeshMotion(C.Structure):
    _fields_ = [
        ("mesh", C.c_uint32),
        ("reserved", C.c_uint32),
        ("positions1", C.POINTER(C.c_float)),
    ]


class RtMaterialDesc(C.Structure):
    _fields_ = [
        ("diffuse_gain", C.c_double),
        ("diffuse_color", c_double3),
        ("diffuse_roughness", C.c_double),
        ("specular_face_color", c_double3),
        ("specular_edge_color", c_double3),
        ("specular_roughness", C.c_double),
        ("specular_ior", C.c_double),
        ("clearcoat_gain", C.c_double),
        ("clearcoat_roughness", C.c_double),
        ("fuzz_gain", C.c_double),
        ("fuzz_color", c_double3),
        ("glass_gain", C.c_double),
        ("glass_ior", C.c_double),
        ("glass_roughness", C.c_double),
        ("refraction_color", c_double3),
        ("glow", c_double3),
        ("presence", C.c_double),
        ("emission", c_double3),
        ("area_light", C.c_int32),
        ("id", C.c_uint32),
        ("subsurface_gain", C.c_double),
        ("subsurface_color", c_double3),
        ("subsurface_dmfp", c_double3),
        ("interior", C.c_int32),
        ("hair", C.c_uint32),
        ("hair_sigma_a", c_double3),
        ("hair_beta_m", C.c_double),
        ("hair_beta_n", C.c_double),
        ("hair_eta", C.c_double),
    ]


class RtCurvesDesc(C.Structure):
    _fields_ = [
        ("p0", C.POINTER(C.c_float)),
        ("p1", C.POINTER(C.c_float)),
        ("v0", C.POINTER(C.c_float)),
        ("v1", C.POINTER(C.c_float)),
        ("n_segments", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


DENSITY_NONE, DENSITY_FBM = 0, 1


class RtMediumDesc(C.Structure):
    _fields_ = [
        ("sigma_a", c_double3),
        ("sigma_s", c_double3),
        ("g", C.c_double),
        ("emission", c_double3),
        ("max_distance", C.c_double),
        ("density", C.c_uint32),
        ("octaves", C.c_uint32),
        ("frequency", C.c_double),
        ("gain", C.c_double),
        ("lacunarity", C.c_double),
        ("coverage", C.c_double),
        ("sharpness", C.c_double),
    ]


class RtLightDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("pad_", C.c_int32),
        ("intensity", C.c_double),
        ("color", c_double3),
        ("p", c_double3),
        ("e1", c_double3),
        ("e2", c_double3),
        ("radius", C.c_double),
    ]


class RtCameraDesc(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("fov_deg", C.c_double),
        ("eye", c_double3),
        ("forward", c_double3),
        ("up", c_double3),
        ("right", c_double3),
        ("lens_radius", C.c_double),
        ("focal_distance", C.c_double),
        ("filter", C.c_int32),
        ("projection", C.c_int32),
        ("filter_width", C.c_double),
        ("ortho_half", C.c_double * 2),
    ]


(PATTERN_CHECKER, PATTERN_FRACTAL, PATTERN_MIX, PATTERN_COLOR_CORRECT, PATTERN_RAMP, PATTERN_TEXTURE,
 PATTERN_TRIPLANAR) = range(7)
WRAP_PERIODIC, WRAP_CLAMP, WRAP_BLACK = range(3)
WRAP_MODES = {"periodic": WRAP_PERIODIC, "clamp": WRAP_CLAMP, "black": WRAP_BLACK}


class RtTextureDesc(C.Structure):
    _fields_ = [("rgb", C.POINTER(C.c_float)), ("width", C.c_uint32), ("height", C.c_uint32)]

# BoundField (src/texture/pattern.rs:238-254), by the RIB parameter names
# (BoundField::from_param, pattern.rs:258-275).
PATTERN_FIELDS = {
    "diffuseColor": 0, "diffuseGain": 1, "diffuseRoughness": 2, "specularFaceColor": 3,
    "specularEdgeColor": 4, "specularRoughness": 5, "clearcoatGain": 6, "fuzzGain": 7, "fuzzColor": 8,
    "glassRefractionGain": 9, "glassRoughness": 10, "refractionColor": 11, "glowColor": 12, "presence": 13,
}
FIELD_PRESENCE = 13


class RtPatternInput(C.Structure):
    _fields_ = [("node", C.c_int32), ("pad_", C.c_int32), ("value", c_double3)]


class RtPatternDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("octaves", C.c_uint32),
        ("color_a", c_double3),
        ("color_b", c_double3),
        ("scale", C.c_double * 2),
        ("frequency", C.c_double),
        ("gain", C.c_double),
        ("lacunarity", C.c_double),
        ("gamma", C.c_double),
        ("saturation", C.c_double),
        ("inputs", RtPatternInput * 3),
        ("ramp_positions", C.POINTER(C.c_double)),
        ("ramp_colors", C.POINTER(C.c_double)),
        ("n_ramp", C.c_uint32),
        ("use_t", C.c_uint32),
        ("texture", C.c_int32),
        ("wrap", C.c_uint32),
        ("udim_tiles", C.POINTER(C.c_uint32)),
        ("udim_textures", C.POINTER(C.c_int32)),
        ("n_udim", C.c_uint32),
        ("udim_reserved", C.c_uint32),
    ]


class RtPatternBinding(C.Structure):
    _fields_ = [("material", C.c_uint32), ("field", C.c_uint32), ("node", C.c_uint32), ("pad_", C.c_uint32)]


class RtIesDesc(C.Structure):
    _fields_ = [
        ("light", C.c_uint32), ("n_v", C.c_uint32), ("n_h", C.c_uint32), ("pad_", C.c_uint32),
        ("v_angles", C.POINTER(C.c_double)), ("h_angles", C.POINTER(C.c_double)),
        ("candela", C.POINTER(C.c_double)), ("world_to_local", C.c_double * 9),
    ]


QUADRIC_SPHERE, QUADRIC_CYLINDER, QUADRIC_CONE, QUADRIC_TORUS, QUADRIC_DISK, QUADRIC_PARABOLOID, \
    QUADRIC_HYPERBOLOID = range(7)


class RtQuadricDesc(C.Structure):
    _fields_ = [("object_to_world", C.c_double * 12), ("params", C.c_double * 8), ("type", C.c_uint32),
                ("material_id", C.c_uint32)]


class RtSceneDesc(C.Structure):
    _fields_ = [
        ("meshes", C.POINTER(RtMeshDesc)),
        ("instances", C.POINTER(RtInstanceDesc)),
        ("materials", C.POINTER(RtMaterialDesc)),
        ("lights", C.POINTER(RtLightDesc)),
        ("n_meshes", C.c_uint32),
        ("n_instances", C.c_uint32),
        ("n_materials", C.c_uint32),
        ("n_lights", C.c_uint32),
        ("camera", RtCameraDesc),
        ("background", c_double3),
        ("env_rgb", C.POINTER(C.c_float)),
        ("env_width", C.c_uint32),
        ("env_height", C.c_uint32),
        ("env_light", C.c_uint32),
        ("env_reserved", C.c_uint32),
        ("patterns", C.POINTER(RtPatternDesc)),
        ("bindings", C.POINTER(RtPatternBinding)),
        ("n_patterns", C.c_uint32),
        ("n_bindings", C.c_uint32),
        ("textures", C.POINTER(RtTextureDesc)),
        ("n_textures", C.c_uint32),
        ("tex_reserved", C.c_uint32),
        ("ies", C.POINTER(RtIesDesc)),
        ("n_ies", C.c_uint32),
        ("ies_reserved", C.c_uint32),
        ("quadrics", C.POINTER(RtQuadricDesc)),
        ("n_quadrics", C.c_uint32),
        ("quadric_reserved", C.c_uint32),
        ("media", C.POINTER(RtMediumDesc)),
        ("n_media", C.c_uint32),
        ("atmosphere", C.c_int32),
        ("curves", C.POINTER(RtCurvesDesc)),
        ("n_curves", C.c_uint32),
        ("curves_reserved", C.c_uint32),
        ("instance_motion", C.POINTER(RtInstanceMotion)),
        ("n_instance_motion", C.c_uint32),
        ("n_mesh_motion", C.c_uint32),
        ("mesh_motion", C.POINTER(RtMeshMotion)),
        ("camera_motion_inv", C.POINTER(C.c_double)),
    ]


class RtParams(C.Structure):
    _fields_ = [
        ("max_depth", C.c_uint32),
        ("rr_start", C.c_uint32),
        ("firefly_clamp", C.c_double),
        ("aovs", C.c_uint32),
        ("guided", C.c_uint32),
        ("guide_fraction", C.c_double),
        ("max_paths", C.c_uint64),
        ("guide_lr", C.c_double),
        ("guide_steps", C.c_uint32),
        ("guide_depth", C.c_uint32),
        ("bvh_build", C.c_uint32),
        ("guide_train_passes", C.c_uint32),
        ("max_trav_steps", C.c_uint32),
        ("wait_polls", C.c_uint32),
    ]


LIGHT_POINT, LIGHT_DISTANT, LIGHT_RECT, LIGHT_SPHERE, LIGHT_DISK, LIGHT_DOME = range(6)
FILTER_BOX, FILTER_TRIANGLE, FILTER_GAUSSIAN = range(3)
PROJECTION_PERSPECTIVE, PROJECTION_ORTHOGRAPHIC = range(2)

for _t, _n in ((RtMeshDesc, 40), (RtInstanceDesc, 104), (RtMaterialDesc, 376), (RtLightDesc, 120),
               (RtCameraDesc, 160), (RtParams, 72), (RtPatternInput, 32), (RtPatternDesc, 264),
               (RtPatternBinding, 16), (RtTextureDesc, 16), (RtIesDesc, 112), (RtQuadricDesc, 168),
               (RtSceneDesc, 392), (RtMediumDesc, 136), (RtCurvesDesc, 40), (RtInstanceMotion, 104),
               (RtMeshMotion, 16)):
    assert C.sizeof(_t) == _n, (_t.__name__, C.sizeof(_t), _n)


def make_params(max_depth=8, rr_start=3, firefly_clamp=60.0, aovs=False, guided=False,
                guide_fraction=0.5, max_paths=0, guide_lr=0.0, guide_steps=0, guide_depth=0, bvh_build="device",
                guide_train_passes=0, max_trav_steps=0, wait_polls=0):
    """Integrator knobs; defaults follow the reference's constants
    (src/raytracer/pt/mod.rs:26-32) except the bounce cap, which the configs set.
    guide_lr / guide_steps: Adam learning rate and steps per sample pass of the
    learned proposal (0 = 1e-2 and 3); guide_depth: only vertices of depth
    below it use the proposal (0 = every depth); guide_train_passes: sample
    passes that train the proposal before it is kept fixed (0 = 512,
    0xFFFFFFFF = never stop). bvh_build: "device" (default) or "host" builds
    the same BVHs on the GPU or on the host cores. max_trav_steps / wait_polls:
    limits of the device's bounded loops (0 = 2^22 traversal steps per ray and
    2^24 polls per tensor-core pipeline wait); a loop that reaches its limit
    ends and the call returns RT_ERR_DEVICE."""
    if bvh_build not in ("device", "host"):
        raise ValueError("bvh_build must be 'device' or 'host'")
    return RtParams(max_depth, rr_start, firefly_clamp, 1 if aovs else 0, 1 if guided else 0,
                    guide_fraction, max_paths, guide_lr, guide_steps, guide_depth,
                    0 if bvh_build == "device" else 1, guide_train_passes, max_trav_steps, wait_polls)
