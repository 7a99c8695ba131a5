"""Host-side scene assembly: numpy arrays in, ``rt_scene_desc`` out.

This is the build-side counterpart of the reference's ``Scene``
(src/scene/mod.rs:27-56) restricted to what the path tracer consumes:
triangle meshes, affine instances, PbrParams materials, lights, camera.
Material helpers follow the reference's legacy mappings
(src/scene/pbr.rs:104-135) and ``PbrParams::default`` (pbr.rs:53-77).
"""
import ctypes as C

import numpy as np

from . import abi

INSTANCE_DTYPE = np.dtype([("xf", "<f8", (12,)), ("mesh", "<u4"), ("mat", "<u4")])
assert INSTANCE_DTYPE.itemsize == C.sizeof(abi.RtInstanceDesc)

IDENTITY_3x4 = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], dtype=np.float64)
# Curve-set handles (add_curves) as instances hold them; the descriptor maps
# them to n_meshes + k, as rt_instance_desc numbers curve sets.
CURVE_BASE = 1 << 30


def _normalize(v):
    v = np.asarray(v, dtype=np.float64)
    n = np.linalg.norm(v)
    return v / n if n > 1e-6 else v


def default_material():
    """PbrParams::default (src/scene/pbr.rs:53-77) with no emission."""
    return dict(diffuse_gain=1.0, diffuse_color=(0.5, 0.5, 0.5), diffuse_roughness=0.0,
                specular_face_color=(0.0, 0.0, 0.0), specular_edge_color=(1.0, 1.0, 1.0),
                specular_roughness=0.2, specular_ior=1.5, clearcoat_gain=0.0,
                clearcoat_roughness=0.1, fuzz_gain=0.0, fuzz_color=(1.0, 1.0, 1.0),
                glass_gain=0.0, glass_ior=1.5, glass_roughness=0.05,
                refraction_color=(1.0, 1.0, 1.0), glow=(0.0, 0.0, 0.0), presence=1.0,
                emission=(0.0, 0.0, 0.0), area_light=-1, id=0, subsurface_gain=0.0,
                subsurface_color=(0.8, 0.6, 0.4), subsurface_dmfp=(0.1, 0.1, 0.1), interior=-1, hair=0,
                hair_sigma_a=(0.0, 0.0, 0.0), hair_beta_m=0.3, hair_beta_n=0.3, hair_eta=1.55)


def matte(color, sigma=0.0, **kw):
    """PbrParams::from_matte (pbr.rs:104-111): diffuse only, specular off
    (specular_ior = 1); `sigma` is the Oren-Nayar roughness."""
    m = default_material()
    m.update(diffuse_gain=1.0, diffuse_color=tuple(color), specular_ior=1.0,
             diffuse_roughness=sigma)
    m.update(kw)
    return m


def ggx_conductor(f0, roughness, **kw):
    """PbrParams::from_metal (pbr.rs:123-131) with a scalar or RGB F0."""
    f0 = (f0, f0, f0) if np.isscalar(f0) else tuple(f0)
    m = default_material()
    m.update(diffuse_gain=0.0, specular_face_color=f0, specular_edge_color=(1.0, 1.0, 1.0),
             specular_roughness=max(roughness, 0.02))
    m.update(kw)
    return m


def ggx_floor(color, roughness, **kw):
    """Diffuse base with a GGX dielectric coat (PbrParams::from_plastic,
    pbr.rs:113-121) at a chosen roughness."""
    m = default_material()
    m.update(diffuse_gain=0.9, diffuse_color=tuple(color), specular_ior=1.5,
             specular_roughness=max(roughness, 0.02))
    m.update(kw)
    return m


def rough_dielectric(ior=1.5, roughness=0.05, **kw):
    """glassRefractionGain = 1 with no diffuse or primary specular lobe."""
    m = default_material()
    m.update(diffuse_gain=0.0, specular_ior=1.0, glass_gain=1.0, glass_ior=ior,
             glass_roughness=roughness)
    m.update(kw)
    return m


def emitter(radiance, area_light=-1, **kw):
    """Black, non-reflecting emitter (no lobes)."""
    m = default_material()
    m.update(diffuse_gain=0.0, specular_ior=1.0, emission=tuple(radiance), area_light=area_light)
    m.update(kw)
    return m


def marschner_hair(color=None, absorption=None, roughness=0.3, azimuthal_roughness=0.3, ior=1.55, **kw):
    """Bxdf "PxrMarschnerHair" (HairParams::from_bxdf_params, hair.rs:82-100):
    absorption given directly or from the fiber colour (pbrt's
    SigmaAFromReflectance); off curves the material is the brown matte the
    reference falls back to (scene_builder.rs:1850-1860)."""
    bn = min(max(azimuthal_roughness, 0.01), 1.0)
    if absorption is None:
        c = np.clip(np.asarray((0.35, 0.2, 0.06) if color is None else color, float), 1e-4, 0.999)
        den = 5.969 - 0.215 * bn + 2.532 * bn ** 2 - 10.73 * bn ** 3 + 5.574 * bn ** 4 + 0.245 * bn ** 5
        absorption = (np.log(c) / den) ** 2
    sa = _rgb(absorption)
    m = matte((0.35, 0.22, 0.12))
    m.update(hair=1, hair_sigma_a=sa, hair_beta_m=float(roughness), hair_beta_n=float(azimuthal_roughness),
             hair_eta=float(ior))
    m.update(kw)
    return m


def volume_hull(**kw):
    """A material that reflects and emits nothing: with an interior medium,
    its surface only bounds the medium (pt/mod.rs:662-680)."""
    m = default_material()
    m.update(diffuse_gain=0.0, specular_ior=1.0)
    m.update(kw)
    return m


def medium(sigma_a, sigma_s, g=0.0, emission=(0.0, 0.0, 0.0), max_distance=np.inf, fbm=None):
    """Medium (src/scene/medium.rs:28-43); `fbm` = dict(frequency, octaves,
    gain, lacunarity, coverage, sharpness) makes it heterogeneous with the
    reference's defaults for missing keys (scene_builder.rs:336-347)."""
    d = dict(sigma_a=_rgb(sigma_a), sigma_s=_rgb(sigma_s), g=float(g), emission=_rgb(emission),
             max_distance=float(max_distance), density=abi.DENSITY_NONE, octaves=0, frequency=0.3,
             gain=0.55, lacunarity=2.0, coverage=0.5, sharpness=4.0)
    if fbm is not None:
        d.update(density=abi.DENSITY_FBM, octaves=5)
        d.update({k: (int(v) if k == "octaves" else float(v)) for k, v in fbm.items()})
    return d


def rot_y(deg):
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], dtype=np.float64)


def affine(linear=None, translate=(0, 0, 0)):
    """Row-major 3x4 object-to-world matrix."""
    m = np.zeros((3, 4), dtype=np.float64)
    m[:, :3] = np.eye(3) if linear is None else linear
    m[:, 3] = translate
    return m.reshape(12)


def _rgb(v):
    if np.ndim(v) == 0:
        return (float(v),) * 3
    return tuple(float(x) for x in v)


class Scene:
    """Scene under construction. Keeps every array alive for as long as the
    descriptor returned by :meth:`desc` is in use."""

    def __init__(self, width, height, fov=40.0):
        self.width, self.height, self.fov = int(width), int(height), float(fov)
        self.meshes = []          # (positions f32 (n,3), indices u32 (m,3), normals or None)
        self.instances = np.zeros(0, dtype=INSTANCE_DTYPE)
        self._inst_chunks = []
        self.materials = []
        self.lights = []
        self.background = (0.0, 0.0, 0.0)
        self.env = None           # (dome light index, (H, W, 3) f32 radiance) or None
        self.mesh_st = {}         # mesh id -> (n, 2) f32 texture coordinates
        self.patterns = []        # pattern nodes (dicts, see add_pattern)
        self.bindings = []        # (material, field id, node)
        self.textures = []        # (H, W, 3) f32 linear RGB base images
        self.ies = {}             # point light index -> (v_angles, h_angles, candela[h][v], world_to_local 3x3)
        self.quadrics = []        # (type, params (<= 8), object_to_world 3x4, material)
        self.media = []           # medium dicts (see medium())
        self.curves = []          # (p0 (n, 4) f32 xyz radius, p1, v0 (n,) f32, v1)
        self.instance_motion = {} # instance -> object_to_world at shutter close (12 f64)
        self.mesh_motion = {}     # mesh id -> (n_vertices, 3) f32 positions at shutter close
        self.camera_motion_inv = None  # 12 f64: Camera::motion_inv (row-major 3x4), or None
        self.atmosphere = -1      # index into media of the global medium, -1 for none
        # Reference default camera: origin, looking down +z (camera.rs:97-103).
        self.eye = np.zeros(3)
        self.forward = np.array([0.0, 0.0, 1.0])
        self.up = np.array([0.0, 1.0, 0.0])
        self.right = np.cross(self.up, self.forward)
        self.lens_radius, self.focal_distance = 0.0, 1.0
        self.filter, self.filter_width = abi.FILTER_BOX, 1.0
        # Camera::projection and ortho_half (camera.rs:80-83, 114): the
        # orthographic window defaults to (aspect, 1).
        self.projection = abi.PROJECTION_PERSPECTIVE
        self.ortho_half = (self.width / max(self.height, 1), 1.0)
        self._desc = None

    # -- geometry --------------------------------------------------------
    def add_mesh(self, positions, indices, normals=None, st=None, positions1=None):
        """Mesh::new(positions, indices, normals, st) (src/geometry/mesh.rs:
        37-60); `st` is (n_vertices, 2) texture coordinates or None;
        `positions1` the vertex positions at shutter close (deformation
        blur, `Mesh::with_motion`, mesh.rs:46-86) or None."""
        p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        i = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
        n = None if normals is None else np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
        if i.size and int(i.max()) >= len(p):
            raise ValueError("mesh index out of range")
        self.meshes.append((p, i, n))
        if positions1 is not None:
            p1 = np.ascontiguousarray(positions1, dtype=np.float32).reshape(-1, 3)
            if p1.shape != p.shape:
                raise ValueError("positions1 needs one position per vertex")
            self.mesh_motion[len(self.meshes) - 1] = p1
        if st is not None:
            st = np.ascontiguousarray(st, dtype=np.float32).reshape(-1, 2)
            if len(st) != len(p):
                raise ValueError("st needs one (s, t) pair per vertex")
            self.mesh_st[len(self.meshes) - 1] = st
        self._desc = None
        return len(self.meshes) - 1

    # -- patterns (src/texture/pattern.rs) ---------------------------------
    # A node input is another node's index (int) or a constant: a float
    # (grey) or an RGB triple. Nodes may read only nodes added before them.
    def _pattern(self, **node):
        self.patterns.append(node)
        self._desc = None
        return len(self.patterns) - 1

    def add_checker(self, color_a, color_b, scale=(1.0, 1.0)):
        """PxrChecker: color_a where floor(s*ss) + floor(t*ts) is even."""
        return self._pattern(type=abi.PATTERN_CHECKER, color_a=_rgb(color_a), color_b=_rgb(color_b),
                             scale=tuple(float(v) for v in scale))

    def add_fractal(self, frequency=1.0, octaves=4, gain=0.5, lacunarity=2.0):
        """PxrFractal: fBm of Perlin noise over world P, remapped to [0, 1]."""
        return self._pattern(type=abi.PATTERN_FRACTAL, frequency=float(frequency), octaves=int(octaves),
                             gain=float(gain), lacunarity=float(lacunarity))

    def add_mix(self, color1, color2, mix):
        """PxrMix: lerp(color1, color2, mix.r)."""
        return self._pattern(type=abi.PATTERN_MIX, inputs=(color1, color2, mix))

    def add_color_correct(self, input, gain=(1, 1, 1), offset=(0, 0, 0), gamma=1.0, saturation=1.0):
        """PxrColorCorrect subset: (in * gain + offset) ^ (1 / gamma), then saturation."""
        return self._pattern(type=abi.PATTERN_COLOR_CORRECT, inputs=(input,), color_a=_rgb(gain),
                             color_b=_rgb(offset), gamma=float(gamma), saturation=float(saturation))

    def add_ramp(self, positions, colors, use_t=False):
        """PxrRamp subset: piecewise-linear colours over s (or t)."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        col = np.ascontiguousarray(colors, dtype=np.float64).reshape(-1, 3)
        if len(pos) != len(col):
            raise ValueError("ramp needs one colour per position")
        return self._pattern(type=abi.PATTERN_RAMP, ramp=(pos, col), use_t=bool(use_t))

    def add_texture(self, rgb):
        """A file texture's base image ((H, W, 3) linear RGB, row 0 at the
        top); returns its index for add_texture_node / add_triplanar."""
        a = np.ascontiguousarray(rgb, dtype=np.float32)
        if a.ndim != 3 or a.shape[2] != 3 or a.shape[0] < 1 or a.shape[1] < 1:
            raise ValueError("texture must be (H, W, 3)")
        self.textures.append(a)
        self._desc = None
        return len(self.textures) - 1

    def add_texture_node(self, texture, wrap="periodic", scale=(1.0, 1.0), udim=None):
        """PxrTexture: the texture at (s, t) * scale, t up (texture row 0 at
        t = 1); `texture` -1 is a missing file (magenta). `udim` = {tile
        number: texture} makes it a UDIM tile set (tile 1001 + s cell + 10 t
        cell, looked up at the cell-local st)."""
        node = dict(type=abi.PATTERN_TEXTURE, texture=int(texture), wrap=abi.WRAP_MODES[wrap],
                    scale=tuple(float(v) for v in scale))
        if udim:
            node["udim"] = {int(k): int(v) for k, v in udim.items()}
        return self._pattern(**node)

    def add_triplanar(self, texture, wrap="periodic", frequency=1.0):
        """Triplanar projection of a texture over world P * frequency,
        blended by the normal's axis weights."""
        return self._pattern(type=abi.PATTERN_TRIPLANAR, texture=int(texture), wrap=abi.WRAP_MODES[wrap],
                             frequency=float(frequency))

    def bind_pattern(self, material, field, node):
        """Material::pattern_bindings: `node`'s output replaces PbrParams
        field `field` (a RIB parameter name such as "diffuseColor", or an
        RT_FIELD_* id) at every shading point."""
        f = abi.PATTERN_FIELDS[field] if isinstance(field, str) else int(field)
        self.bindings.append((int(material), f, int(node)))
        self._desc = None

    def add_curves(self, p0, p1, v0, v1):
        """A curve set (src/geometry/curves.rs:15-26): rounded-cone segments
        from p0 to p1 (rows xyz + radius) with curve parameters v0, v1.
        Returns a handle that add_instance places like a mesh id."""
        p0 = np.ascontiguousarray(np.reshape(p0, (-1, 4)), dtype=np.float32)
        p1 = np.ascontiguousarray(np.reshape(p1, (-1, 4)), dtype=np.float32)
        v0 = np.ascontiguousarray(np.ravel(v0), dtype=np.float32)
        v1 = np.ascontiguousarray(np.ravel(v1), dtype=np.float32)
        if not (len(p0) == len(p1) == len(v0) == len(v1)):
            raise ValueError("curve arrays of different lengths")
        self.curves.append((p0, p1, v0, v1))
        self._desc = None
        return CURVE_BASE + len(self.curves) - 1

    def add_instance(self, mesh_id, material_id, xform=None, xform1=None):
        """Instance of a mesh or curve set; `xform1` is its object-to-world
        transform at shutter close (transform motion blur,
        `Instance::with_motion`, mesh.rs:244-253) or None."""
        rec = np.zeros(1, dtype=INSTANCE_DTYPE)
        rec["xf"][0] = IDENTITY_3x4 if xform is None else np.asarray(xform, dtype=np.float64).reshape(12)
        rec["mesh"][0] = mesh_id
        rec["mat"][0] = material_id
        self._inst_chunks.append(rec)
        self._desc = None
        if xform1 is not None:
            self.instance_motion[self.n_instances - 1] = np.asarray(xform1, dtype=np.float64).reshape(12).copy()
        return self.n_instances - 1

    @property
    def has_motion(self):
        """scene_builder.rs:239-241: rays draw a shutter time."""
        return bool(self.instance_motion or self.mesh_motion or self.camera_motion_inv is not None)

    def add_instances(self, mesh_ids, material_ids, xforms):
        """Vectorised instance placement: xforms (n, 12) row-major 3x4."""
        n = len(mesh_ids)
        rec = np.zeros(n, dtype=INSTANCE_DTYPE)
        rec["xf"] = np.asarray(xforms, dtype=np.float64).reshape(n, 12)
        rec["mesh"] = mesh_ids
        rec["mat"] = material_ids
        self._inst_chunks.append(rec)
        self._desc = None

    @property
    def n_instances(self):
        return sum(len(c) for c in self._inst_chunks)

    def add_material(self, m):
        self.materials.append(dict(m))
        self._desc = None
        return len(self.materials) - 1

    # -- lights ----------------------------------------------------------
    def _light(self, type_, intensity, color, p=(0, 0, 0), e1=(0, 0, 0), e2=(0, 0, 0), radius=0.0):
        self.lights.append(dict(type=type_, intensity=float(intensity), color=tuple(color),
                                p=tuple(p), e1=tuple(e1), e2=tuple(e2), radius=float(radius)))
        self._desc = None
        return len(self.lights) - 1

    def add_quadric(self, kind, params, material, object_to_world=None):
        """An analytic RiSpec quadric (rt_quadric_desc): `kind` one of
        abi.QUADRIC_*, `params` as rt_scene.h lists them per kind."""
        xf = affine() if object_to_world is None else np.asarray(object_to_world, np.float64).reshape(3, 4)
        pr = [float(v) for v in params]
        if len(pr) > 8:
            raise ValueError("at most 8 quadric parameters")
        self.quadrics.append((int(kind), pr + [0.0] * (8 - len(pr)), xf.copy(), int(material)))
        self._desc = None
        return len(self.quadrics) - 1

    def add_medium(self, med, atmosphere=False):
        """A participating medium (see medium()); materials reference it by
        their `interior` index, or it becomes the scene's atmosphere."""
        self.media.append(dict(med))
        if atmosphere:
            self.atmosphere = len(self.media) - 1
        self._desc = None
        return len(self.media) - 1

    def add_point_light(self, position, intensity, color=(1, 1, 1), ies=None, world_to_local=None):
        """Light::point; `ies` = (vertical angles, horizontal angles,
        candela[h][v]) reshapes its output (src/scene/ies.rs), oriented by
        `world_to_local` (3x3, identity by default: 0 degrees points down -y)."""
        li = self._light(abi.LIGHT_POINT, intensity, color, p=position)
        if ies is not None:
            v, h, c = (np.ascontiguousarray(a, dtype=np.float64) for a in ies)
            if c.shape != (len(h), len(v)) or len(v) == 0 or len(h) == 0:
                raise ValueError("ies candela must be (n_h, n_v)")
            m = np.eye(3) if world_to_local is None else np.asarray(world_to_local, np.float64).reshape(3, 3)
            self.ies[li] = (v, h, np.ascontiguousarray(c), np.ascontiguousarray(m))
        return li

    def add_distant_light(self, direction, intensity, color=(1, 1, 1), angular_radius=0.0):
        return self._light(abi.LIGHT_DISTANT, intensity, color, e1=direction, radius=angular_radius)

    def add_dome_light(self, intensity, color=(1, 1, 1), env=None):
        """Light::dome (src/scene/light.rs:142-151): radiance color *
        intensity from every direction, times the lat-long environment map
        `env` ((H, W, 3) float radiance, row 0 at +y) when one is given
        (one map per scene)."""
        li = self._light(abi.LIGHT_DOME, intensity, color)
        if env is not None:
            self.env = (li, np.ascontiguousarray(env, dtype=np.float32).reshape(np.shape(env)[0], -1, 3))
        return li

    def add_rect_light(self, corner, edge1, edge2, intensity, color=(1, 1, 1)):
        return self._light(abi.LIGHT_RECT, intensity, color, p=corner, e1=edge1, e2=edge2)

    def add_emissive_quad(self, corner, edge1, edge2, radiance):
        """A sampleable rectangle light plus its emissive geometry, as the
        reference's scene builder makes for an AreaLightSource Polygon
        (src/parser/scene_builder.rs:924-933)."""
        corner, e1, e2 = (np.asarray(v, dtype=np.float64) for v in (corner, edge1, edge2))
        li = self.add_rect_light(corner, e1, e2, 1.0, radiance)
        mat = self.add_material(emitter(radiance, area_light=li))
        pos = np.array([corner, corner + e1, corner + e1 + e2, corner + e2])
        mesh = self.add_mesh(pos, [[0, 1, 2], [0, 2, 3]])
        self.add_instance(mesh, mat)
        return li

    # -- camera ----------------------------------------------------------
    def look_at(self, eye, target, up=(0, 1, 0), fov=None):
        """Camera::set_transform (src/scene/camera.rs:124-129)."""
        self.eye = np.asarray(eye, dtype=np.float64)
        self.forward = _normalize(np.asarray(target, dtype=np.float64) - self.eye)
        self.right = _normalize(np.cross(self.forward, np.asarray(up, dtype=np.float64)))
        self.up = _normalize(np.cross(self.right, self.forward))
        if fov is not None:
            self.fov = float(fov)
        self._desc = None

    # -- descriptor ------------------------------------------------------
    def triangle_count(self):
        """Effective (instanced) triangles."""
        inst = self.instance_array()
        per_mesh = np.array([len(m[1]) for m in self.meshes], dtype=np.int64)
        mesh = inst["mesh"][inst["mesh"] < CURVE_BASE] if len(inst) else inst["mesh"]
        return int(per_mesh[mesh].sum()) if len(mesh) else 0

    def instance_array(self):
        if self._inst_chunks:
            if len(self._inst_chunks) > 1:
                self._inst_chunks = [np.concatenate(self._inst_chunks)]
            return self._inst_chunks[0]
        return np.zeros(0, dtype=INSTANCE_DTYPE)

    def desc(self):
        if self._desc is not None:
            return self._desc
        keep = []
        mesh_arr = (abi.RtMeshDesc * max(1, len(self.meshes)))()
        for k, (p, i, n) in enumerate(self.meshes):
            keep += [p, i, n]
            st = self.mesh_st.get(k)
            if st is not None:
                keep.append(st)
                mesh_arr[k].st = st.ctypes.data_as(C.POINTER(C.c_float))
            mesh_arr[k].positions = p.ctypes.data_as(C.POINTER(C.c_float))
            mesh_arr[k].indices = i.ctypes.data_as(C.POINTER(C.c_uint32))
            mesh_arr[k].normals = n.ctypes.data_as(C.POINTER(C.c_float)) if n is not None else None
            mesh_arr[k].n_vertices = len(p)
            mesh_arr[k].n_triangles = len(i)
        inst = np.ascontiguousarray(self.instance_array())
        if len(inst) and (inst["mesh"] >= CURVE_BASE).any():
            inst = inst.copy()
            cm = inst["mesh"] >= CURVE_BASE
            inst["mesh"][cm] = inst["mesh"][cm] - CURVE_BASE + len(self.meshes)
        keep.append(inst)
        mat_arr = (abi.RtMaterialDesc * max(1, len(self.materials)))()
        for k, m in enumerate(self.materials):
            for key, val in m.items():
                if isinstance(val, tuple):
                    setattr(mat_arr[k], key, abi.c_double3(*val))
                else:
                    setattr(mat_arr[k], key, val)
        light_arr = (abi.RtLightDesc * max(1, len(self.lights)))()
        for k, l in enumerate(self.lights):
            light_arr[k].type = l["type"]
            light_arr[k].intensity = l["intensity"]
            light_arr[k].color = abi.c_double3(*l["color"])
            light_arr[k].p = abi.c_double3(*l["p"])
            light_arr[k].e1 = abi.c_double3(*l["e1"])
            light_arr[k].e2 = abi.c_double3(*l["e2"])
            light_arr[k].radius = l["radius"]
        cam = abi.RtCameraDesc(self.width, self.height, self.fov, abi.c_double3(*self.eye),
                               abi.c_double3(*self.forward), abi.c_double3(*self.up),
                               abi.c_double3(*self.right), self.lens_radius, self.focal_distance,
                               self.filter, self.projection, self.filter_width,
                               (C.c_double * 2)(*self.ortho_half))
        d = abi.RtSceneDesc()
        d.meshes = mesh_arr
        d.instances = inst.ctypes.data_as(C.POINTER(abi.RtInstanceDesc))
        d.materials = mat_arr
        d.lights = light_arr
        d.n_meshes, d.n_instances = len(self.meshes), len(inst)
        d.n_materials, d.n_lights = len(self.materials), len(self.lights)
        d.camera = cam
        d.background = abi.c_double3(*self.background)
        if self.env is not None:
            li, env = self.env
            keep.append(env)
            d.env_rgb = env.ctypes.data_as(C.POINTER(C.c_float))
            d.env_height, d.env_width = env.shape[0], env.shape[1]
            d.env_light = li
        pat_arr = (abi.RtPatternDesc * max(1, len(self.patterns)))()
        for k, node in enumerate(self.patterns):
            pd = pat_arr[k]
            pd.type = node["type"]
            pd.octaves = node.get("octaves", 0)
            pd.color_a = abi.c_double3(*node.get("color_a", (0, 0, 0)))
            pd.color_b = abi.c_double3(*node.get("color_b", (0, 0, 0)))
            pd.scale = (C.c_double * 2)(*node.get("scale", (1.0, 1.0)))
            pd.frequency, pd.gain = node.get("frequency", 1.0), node.get("gain", 0.5)
            pd.lacunarity = node.get("lacunarity", 2.0)
            pd.gamma, pd.saturation = node.get("gamma", 1.0), node.get("saturation", 1.0)
            for j, v in enumerate(node.get("inputs", ())):
                if isinstance(v, (int, np.integer)) and not isinstance(v, bool):
                    pd.inputs[j].node = int(v)
                else:
                    pd.inputs[j].node = -1
                    pd.inputs[j].value = abi.c_double3(*_rgb(v))
            for j in range(len(node.get("inputs", ())), 3):
                pd.inputs[j].node = -1
            if "ramp" in node:
                pos, col = node["ramp"]
                keep += [pos, col]
                pd.ramp_positions = pos.ctypes.data_as(C.POINTER(C.c_double))
                pd.ramp_colors = col.ctypes.data_as(C.POINTER(C.c_double))
                pd.n_ramp = len(pos)
                pd.use_t = int(node["use_t"])
            pd.texture = node.get("texture", -1)
            pd.wrap = node.get("wrap", 0)
            if node.get("udim"):
                tiles = np.array(sorted(node["udim"]), dtype=np.uint32)
                texs = np.array([node["udim"][int(t)] for t in tiles], dtype=np.int32)
                keep += [tiles, texs]
                pd.udim_tiles = tiles.ctypes.data_as(C.POINTER(C.c_uint32))
                pd.udim_textures = texs.ctypes.data_as(C.POINTER(C.c_int32))
                pd.n_udim = len(tiles)
        bind_arr = (abi.RtPatternBinding * max(1, len(self.bindings)))()
        for k, (m, f, n) in enumerate(self.bindings):
            bind_arr[k].material, bind_arr[k].field, bind_arr[k].node = m, f, n
        if self.patterns:
            d.patterns = pat_arr
            d.n_patterns = len(self.patterns)
        if self.bindings:
            d.bindings = bind_arr
            d.n_bindings = len(self.bindings)
        tex_arr = (abi.RtTextureDesc * max(1, len(self.textures)))()
        for k, t in enumerate(self.textures):
            keep.append(t)
            tex_arr[k].rgb = t.ctypes.data_as(C.POINTER(C.c_float))
            tex_arr[k].height, tex_arr[k].width = t.shape[0], t.shape[1]
        if self.textures:
            d.textures = tex_arr
            d.n_textures = len(self.textures)
        self._desc = d
        ies_arr = (abi.RtIesDesc * max(1, len(self.ies)))()
        for k, (li, (v, h, c, m)) in enumerate(sorted(self.ies.items())):
            keep += [v, h, c]
            e = ies_arr[k]
            e.light, e.n_v, e.n_h = li, len(v), len(h)
            e.v_angles = v.ctypes.data_as(C.POINTER(C.c_double))
            e.h_angles = h.ctypes.data_as(C.POINTER(C.c_double))
            e.candela = c.ctypes.data_as(C.POINTER(C.c_double))
            e.world_to_local = (C.c_double * 9)(*m.reshape(9))
        if self.ies:
            d.ies = ies_arr
            d.n_ies = len(self.ies)
        quad_arr = (abi.RtQuadricDesc * max(1, len(self.quadrics)))()
        for k, (kind, pr, xf, mat) in enumerate(self.quadrics):
            q = quad_arr[k]
            q.object_to_world = (C.c_double * 12)(*xf.reshape(12))
            q.params = (C.c_double * 8)(*pr)
            q.type, q.material_id = kind, mat
        if self.quadrics:
            d.quadrics = quad_arr
            d.n_quadrics = len(self.quadrics)
        med_arr = (abi.RtMediumDesc * max(1, len(self.media)))()
        for k, m in enumerate(self.media):
            for key, val in m.items():
                setattr(med_arr[k], key, abi.c_double3(*val) if isinstance(val, tuple) else val)
        if self.media:
            d.media = med_arr
            d.n_media = len(self.media)
        d.atmosphere = self.atmosphere
        cur_arr = (abi.RtCurvesDesc * max(1, len(self.curves)))()
        for k, (p0, p1, v0, v1) in enumerate(self.curves):
            keep += [p0, p1, v0, v1]
            c = cur_arr[k]
            c.p0, c.p1 = (a.ctypes.data_as(C.POINTER(C.c_float)) for a in (p0, p1))
            c.v0, c.v1 = (a.ctypes.data_as(C.POINTER(C.c_float)) for a in (v0, v1))
            c.n_segments = len(v0)
        if self.curves:
            d.curves = cur_arr
            d.n_curves = len(self.curves)
        im_arr = (abi.RtInstanceMotion * max(1, len(self.instance_motion)))()
        for k, (ii, xf1) in enumerate(sorted(self.instance_motion.items())):
            im_arr[k].instance = ii
            im_arr[k].object_to_world1 = (C.c_double * 12)(*xf1)
        if self.instance_motion:
            d.instance_motion = im_arr
            d.n_instance_motion = len(self.instance_motion)
        mm_arr = (abi.RtMeshMotion * max(1, len(self.mesh_motion)))()
        for k, (mi, p1) in enumerate(sorted(self.mesh_motion.items())):
            keep.append(p1)
            mm_arr[k].mesh = mi
            mm_arr[k].positions1 = p1.ctypes.data_as(C.POINTER(C.c_float))
        if self.mesh_motion:
            d.mesh_motion = mm_arr
            d.n_mesh_motion = len(self.mesh_motion)
        cam_mot = None
        if self.camera_motion_inv is not None:
            cam_mot = (C.c_double * 12)(*np.asarray(self.camera_motion_inv, dtype=np.float64).reshape(12))
            d.camera_motion_inv = cam_mot
        self._keep = (keep, mesh_arr, mat_arr, light_arr, pat_arr, bind_arr, tex_arr, ies_arr, quad_arr, med_arr,
                      cur_arr, im_arr, mm_arr, cam_mot)
        return d
