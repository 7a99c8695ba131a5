"""RIB scene files -> rtcuda scenes (the reference's ``parse_rib_bytes`` +
``SceneBuilder::build``, src/parser/parser.rs, src/parser/binary.rs and
src/parser/scene_builder.rs), text or binary RIB, for the part of RenderMan the CUDA path
renders: triangle meshes and polygons, quadrics, instancing, legacy and
PxrSurface materials, point / distant / area lights, the camera.

Same conventions as the reference: requests are an identifier followed by
values (numbers, strings, or homogeneous [arrays]); ``#`` starts a comment;
parameter tokens match on their last word ("uniform float roughness");
the current transform keeps the pre-WorldBegin camera transform, so world
geometry lands in camera space and the camera sits at the origin looking
down +z; ``Translate`` / ``Rotate`` / ``Scale`` / ``ConcatTransform``
post-multiply the current matrix (column vectors); RIB matrices are
transposed on ingest (scene_builder.rs:1925-1938); ``LightSource``
positions are taken as written, without the current transform
(scene_builder.rs:1582-1635).

Deviations (recorded in ``RibScene.warnings`` at load time):
  * Quadrics (Sphere, Cylinder, Cone, Disk, Torus, Paraboloid,
    Hyperboloid) and the emitter shapes of PxrSphereLight / PxrDiskLight
    are analytic quadrics, as the reference's objects; inside ObjectBegin
    they are skipped, as the reference does.
  * Bilinear / bicubic PatchMesh and Patch are diced by the current
    Basis, as the reference does, NuPatch NURBS untrimmed;
    SubdivisionMesh, GeneralPolygon and motion blur are skipped with a
    warning (motion blocks use their first sample); Curves and Points
    become curve sets (rounded-cone segments) and PxrMarschnerHair their
    hair material; Interior and Atmosphere media (homogeneous or fBm) and
    PxrSurface subsurface parameters are carried; Displace "noise" moves polygon-mesh vertices at load time as
    the reference does; a PxrDomeLight lightColorMap is read when it is a
    Radiance .hdr (one map per scene).
  * Pattern graphs: PxrChecker, PxrFractal, PxrMix, PxrColorCorrect,
    PxrRamp, PxrTexture and triplanar nodes and Bxdf "reference"
    connections are carried, UDIM tile sets included; texture files are
    read when they are .tex, Radiance .hdr or PNG (others render magenta,
    as the reference's unreadable files do); presence connections are
    skipped.
    Tessellated quadrics carry the reference's st, hyperboloids excepted.
"""
import math
import os

import numpy as np

from . import abi
from .scene import Scene, default_material, emitter, marschner_hair, medium

# ---- parsing (src/parser/parser.rs) --------------------------------------------------------


class RibError(ValueError):
    pass


def _skip_ws(s, i):
    n = len(s)
    while i < n:
        c = s[i]
        if c in " \t\r\n\f\v":
            i += 1
        elif c == "#":
            j = s.find("\n", i)
            i = n if j < 0 else j
        else:
            break
    return i


def _string(s, i):
    j = s.find('"', i + 1)
    if j < 0:
        raise RibError("unterminated string")
    return s[i + 1:j], j + 1


_NUM_CHARS = set("0123456789+-.eE")


def _number(s, i):
    j = i
    n = len(s)
    while j < n and s[j] in _NUM_CHARS:
        j += 1
    try:
        return float(s[i:j]), j
    except ValueError:
        raise RibError(f"bad number near {s[i:i + 20]!r}") from None


def parse_rib(text):
    """List of (name, values); values are float, str, list of floats or list
    of strings."""
    out = []
    i = _skip_ws(text, 0)
    n = len(text)
    while i < n:
        j = i
        while j < n and (text[j].isascii() and text[j].isalpha() or text[j] == "_"):
            j += 1
        if j == i:
            raise RibError(f"failed to parse RIB near: {text[i:i + 60]!r}")
        name = text[i:j]
        vals = []
        i = _skip_ws(text, j)
        while i < n:
            c = text[i]
            if c == '"':
                v, i = _string(text, i)
                vals.append(v)
            elif c == "[":
                i = _skip_ws(text, i + 1)
                if i < n and text[i] == '"':
                    arr = []
                    while True:
                        i = _skip_ws(text, i)
                        if i >= n:
                            raise RibError("unterminated array")
                        if text[i] == "]":
                            i += 1
                            break
                        v, i = _string(text, i)
                        arr.append(v)
                    vals.append(arr)
                else:
                    arr = []
                    while True:
                        i = _skip_ws(text, i)
                        if i >= n:
                            raise RibError("unterminated array")
                        if text[i] == "]":
                            i += 1
                            break
                        v, i = _number(text, i)
                        arr.append(v)
                    vals.append([float(x) for x in arr])
            elif c.isdigit() or c in "+-.":
                v, i = _number(text, i)
                vals.append(v)
            else:
                break
            i = _skip_ws(text, i)
        out.append((name, vals))
    return out


# ---- binary RIB (src/parser/binary.rs: RISpec 3.2 Appendix C.2) ----------------------------


def looks_binary(data):
    """True when bytes >= 0200 appear outside comments (binary.rs:21-33)."""
    in_comment = False
    for b in data:
        if b == 0x23:
            in_comment = True
        elif b == 0x0A:
            in_comment = False
        elif b >= 0x80 and not in_comment:
            return True
    return False


def _be_uint(data, pos, n):
    if pos + n > len(data):
        raise RibError(f"binary RIB: truncated integer at byte {pos}")
    return int.from_bytes(data[pos:pos + n], "big"), pos + n


def _be_int(data, pos, n):
    v, pos = _be_uint(data, pos, n)
    if v >> (8 * n - 1):
        v -= 1 << (8 * n)
    return v, pos


def _bin_string(data, pos):
    if pos >= len(data):
        raise RibError("binary RIB: truncated string")
    code = data[pos]
    pos += 1
    if 0x90 <= code <= 0x9F:
        n = code - 0x90
    elif 0xA0 <= code <= 0xA3:
        n, pos = _be_uint(data, pos, code - 0xA0 + 1)
    else:
        raise RibError(f"binary RIB: expected string code, got {code:#o}")
    if pos + n > len(data):
        raise RibError("binary RIB: truncated string body")
    return data[pos:pos + n].decode("utf-8", errors="replace"), pos + n


def decode_binary(data):
    """Binary RIB bytes -> canonical text RIB (binary.rs:86-198): integers
    0200-0203, fixed point 0204-0217, strings 0220-0243, float 0244, double
    0245, request use 0246, string-token definitions 0310-0313, request
    definition 0314, string-token references 0315-0316; other codes >= 0200
    are skipped."""
    out = []
    requests, strings = {}, {}
    pos, n = 0, len(data)
    quote = lambda t: '"' + t.replace("\\", "\\\\").replace('"', '\\"').replace("\n", "\\n") + '"'
    while pos < n:
        b = data[pos]
        if b < 0x80:
            if b == 0x23:
                j = data.find(b"\n", pos)
                j = n if j < 0 else j
                out.append(data[pos:j].decode("latin-1"))
                pos = j
            else:
                out.append(chr(b))
                pos += 1
        elif b <= 0x83:
            v, pos = _be_int(data, pos + 1, b - 0x80 + 1)
            out.append(f" {v} ")
        elif b <= 0x8F:
            q = b - 0x84
            d, w = q // 4, q % 4
            raw, pos = _be_int(data, pos + 1, w + 1 + d)
            out.append(f" {repr(raw / 256.0 ** d)} ")
        elif b <= 0xA3:
            t, pos = _bin_string(data, pos)
            out.append(" " + quote(t) + " ")
        elif b == 0xA4:
            raw, pos = _be_uint(data, pos + 1, 4)
            out.append(f" {str(np.frombuffer(raw.to_bytes(4, 'little'), '<f4')[0])} ")  # shortest f32 form
        elif b == 0xA5:
            raw, pos = _be_uint(data, pos + 1, 8)
            out.append(f" {repr(float(np.frombuffer(raw.to_bytes(8, 'little'), '<f8')[0]))} ")
        elif b == 0xA6:
            if pos + 1 >= n:
                raise RibError("binary RIB: truncated request code")
            code = data[pos + 1]
            pos += 2
            if code not in requests:
                raise RibError(f"binary RIB: request code {code} used before definition")
            out.append(f"\n{requests[code]} ")
        elif 0xC8 <= b <= 0xCB:
            tok, pos = _be_uint(data, pos + 1, b - 0xC8 + 1)
            strings[tok], pos = _bin_string(data, pos)
        elif b == 0xCC:
            if pos + 1 >= n:
                raise RibError("binary RIB: truncated request def")
            code = data[pos + 1]
            requests[code], pos = _bin_string(data, pos + 2)
        elif b in (0xCD, 0xCE):
            tok, pos = _be_uint(data, pos + 1, b - 0xCD + 1)
            if tok not in strings:
                raise RibError(f"binary RIB: string token {tok} used before definition")
            out.append(" " + quote(strings[tok]) + " ")
        else:
            pos += 1
    return "".join(out)


def _as_number(v):
    if isinstance(v, float):
        return v
    if isinstance(v, list) and len(v) == 1 and isinstance(v[0], float):
        return v[0]
    return None


def _as_numbers(v):
    if isinstance(v, float):
        return [v]
    if isinstance(v, list) and all(isinstance(x, float) for x in v):
        return v
    return None


def _as_str(v):
    if isinstance(v, str):
        return v
    if isinstance(v, list) and len(v) == 1 and isinstance(v[0], str):
        return v[0]
    return None


class _Params:
    """Token/value pairs from a value index on (ast.rs:63-112)."""

    def __init__(self, vals, start):
        self.pairs = []
        i = start
        while i + 1 < len(vals):
            t = _as_str(vals[i])
            if t is None:
                break
            self.pairs.append((t, vals[i + 1]))
            i += 2

    def get(self, name):
        for t, v in self.pairs:
            w = t.split()
            if w and w[-1] == name:
                return v
        return None

    def number(self, name):
        v = self.get(name)
        return None if v is None else _as_number(v)

    def numbers(self, name):
        v = self.get(name)
        return None if v is None else _as_numbers(v)

    def string(self, name):
        v = self.get(name)
        return None if v is None else _as_str(v)


def _or(v, default):
    return default if v is None else v


def dice_curve(ctrl, cubic, w_root, w_tip, segs):
    """dice_curve (curves.rs:193-247): sample the curve (each cubic span of
    the basis at `segs` steps, the last span including its end; linear
    curves at their control points), then one rounded-cone segment per
    pair of samples with the half-width going linearly root to tip and v
    = sample index / (samples - 1). Returns (p0, p1, v0, v1) or None."""
    from .patches import basis_weights
    ctrl = np.asarray(ctrl, np.float64)
    if cubic is None:
        pts = ctrl
    else:
        m, step = cubic
        n = len(ctrl)
        if n < 4:
            return None
        spans = (n - 4) // step + 1
        pts = []
        for sp in range(spans):
            g = ctrl[sp * step:sp * step + 4]
            count = segs + 1 if sp == spans - 1 else segs
            pts.append(basis_weights(m, np.arange(count) / segs) @ g)
        pts = np.concatenate(pts)
    if len(pts) < 2:
        return None
    v = np.arange(len(pts)) / (len(pts) - 1)
    r = (w_root + (w_tip - w_root) * v) * 0.5
    p = np.concatenate([pts, r[:, None]], axis=1)
    return p[:-1], p[1:], v[:-1], v[1:]


def _num(vals, k):
    return _as_number(vals[k]) if k < len(vals) else None


def _str(vals, k):
    return _as_str(vals[k]) if k < len(vals) else None


# ---- matrices (src/math/matrix.rs; column-vector convention) --------------------------------


def _translate(x, y, z):
    m = np.eye(4)
    m[:3, 3] = (x, y, z)
    return m


def _scale(x, y, z):
    return np.diag([x, y, z, 1.0])


def _rotate(angle, x, y, z):
    a = np.array([x, y, z], dtype=np.float64)
    ln = np.linalg.norm(a)
    if ln > 1e-6:
        a = a / ln
    x, y, z = a
    r = math.radians(angle)
    c, s = math.cos(r), math.sin(r)
    t = 1.0 - c
    m = np.eye(4)
    m[:3, :3] = [[c + x * x * t, x * y * t - z * s, x * z * t + y * s],
                 [y * x * t + z * s, c + y * y * t, y * z * t - x * s],
                 [z * x * t - y * s, z * y * t + x * s, c + z * z * t]]
    return m


def _from_rib(v):
    return np.array(v, dtype=np.float64).reshape(4, 4).T


def _xf_point(m, p):
    q = m @ np.array([p[0], p[1], p[2], 1.0])
    return q[:3] / q[3] if abs(q[3] - 1.0) >= 1e-6 else q[:3]


def _xf_vec(m, v):
    return m[:3, :3] @ np.asarray(v, dtype=np.float64)


MAX_ARCHIVE_DEPTH = 16

# ---- quadrics --------------------------------------------------------------------------------
# Arguments per request (scene_builder.rs:813-909); each becomes an analytic
# quadric (rt_quadric_desc) with the same parameters.
_QUADRIC_ARGS = {"Sphere": 4, "Cylinder": 4, "Cone": 3, "Disk": 3, "Torus": 5, "Paraboloid": 4, "Hyperboloid": 7}
_QUADRIC_KIND = {"Sphere": abi.QUADRIC_SPHERE, "Cylinder": abi.QUADRIC_CYLINDER, "Cone": abi.QUADRIC_CONE,
                 "Disk": abi.QUADRIC_DISK, "Torus": abi.QUADRIC_TORUS, "Paraboloid": abi.QUADRIC_PARABOLOID,
                 "Hyperboloid": abi.QUADRIC_HYPERBOLOID}

# ---- materials (src/scene/material.rs, src/scene/pbr.rs) ------------------------------------


def _pbr_matte(c):
    m = default_material()
    m.update(diffuse_gain=1.0, diffuse_color=tuple(c), specular_ior=1.0)
    return m


def _pbr_plastic(c, rough):
    m = default_material()
    m.update(diffuse_gain=0.9, diffuse_color=tuple(c), specular_ior=1.5, specular_roughness=max(rough, 0.02))
    return m


def _pbr_metal(c, rough):
    m = default_material()
    m.update(diffuse_gain=0.0, specular_face_color=tuple(c), specular_edge_color=(1.0, 1.0, 1.0),
             specular_roughness=max(rough, 0.02))
    return m


def _pbr_bxdf(p):
    """PbrParams::from_bxdf_params (pbr.rs:133-187)."""
    m = default_material()
    m.update(diffuse_gain=1.0, diffuse_color=(0.18, 0.18, 0.18), specular_ior=1.5, specular_roughness=0.2)
    colors = {"diffuseColor": "diffuse_color", "specularFaceColor": "specular_face_color",
              "specularEdgeColor": "specular_edge_color", "fuzzColor": "fuzz_color",
              "refractionColor": "refraction_color"}
    scalars = {"diffuseGain": "diffuse_gain", "diffuseRoughness": "diffuse_roughness",
               "specularRoughness": "specular_roughness", "specularIor": "specular_ior",
               "clearcoatGain": "clearcoat_gain", "clearcoatRoughness": "clearcoat_roughness",
               "fuzzGain": "fuzz_gain", "glassRefractionGain": "glass_gain", "glassIor": "glass_ior",
               "glassRoughness": "glass_roughness", "presence": "presence"}
    for tok, key in colors.items():
        v = p.numbers(tok)
        if v is not None and len(v) >= 3:
            m[key] = tuple(v[:3])
    for tok, key in scalars.items():
        v = p.number(tok)
        if v is not None:
            m[key] = v
    # Subsurface walk (pbr.rs:174-183): a scalar mean free path applies to
    # all three channels.
    v = p.number("subsurfaceGain")
    if v is not None:
        m["subsurface_gain"] = v
    v = p.numbers("subsurfaceColor")
    if v is not None and len(v) >= 3:
        m["subsurface_color"] = tuple(v[:3])
    v = p.numbers("subsurfaceDmfp")
    if v:
        m["subsurface_dmfp"] = tuple(v[:3]) if len(v) >= 3 else (v[0],) * 3
    gg = p.number("glowGain") or 0.0
    gc = p.numbers("glowColor")
    gc = tuple(gc[:3]) if gc is not None and len(gc) >= 3 else (1.0, 1.0, 1.0)
    m["glow"] = tuple(c * gg for c in gc)
    for key in ("specular_roughness", "glass_roughness", "clearcoat_roughness"):
        m[key] = min(max(m[key], 0.005), 1.0)
    return m


class _State:
    def __init__(self):
        self.color = (1.0, 1.0, 1.0)
        self.surface = "matte"
        self.roughness = 0.1
        self.area_light = None   # (intensity, color)
        self.bxdf = None         # material dict
        self.bxdf_bindings = []  # (field id, pattern node) of the active Bxdf
        self.displace = None     # Displace "noise" parameters (dict) for tessellated meshes
        self.shading_rate = 1.0  # sets the patch dicing
        self.basis_u = ("bezier", None)  # Basis: (name or 16 numbers, step or None) per direction
        self.basis_v = ("bezier", None)
        self.identifier = None
        self.interior = -1       # Interior medium bound to subsequent geometry
        self.hair = None         # Bxdf "PxrMarschnerHair" parameters (dict)
        self.motion_t0 = None    # transform-motion endpoints of a closed MotionBegin block (4x4)
        self.motion_t1 = None

    def copy(self):
        s = _State()
        s.__dict__.update(self.__dict__)
        return s


class RibScene(Scene):
    """An rtcuda Scene built from a RIB file; ``pixel_samples`` and
    ``warnings`` as the reference's Scene keeps them."""

    def __init__(self, width, height, fov):
        super().__init__(width, height, fov)
        self.pixel_samples = (1, 1)
        self.warnings = []

    @property
    def spp(self):
        return self.pixel_samples[0] * self.pixel_samples[1]


class _Builder:
    def __init__(self, base_dir=None):
        self.width, self.height, self.fov = 640, 480, 45.0
        self.dof = None
        self.projection = abi.PROJECTION_PERSPECTIVE
        self.screen_window = None
        self.filter = (abi.FILTER_BOX, 1.0)
        self.pixel_samples = (1, 1)
        self.background = (0.0, 0.0, 0.0)
        self.state = _State()
        self.attr_stack = []
        self.xf = [np.eye(4)]
        self.base_dir = base_dir
        self.archives = {}
        self.recording = None
        self.object_defs = {}
        self.defining = None
        self.archive_depth = 0
        self.object_ids = {}
        self.next_id = 1
        self.warned = []
        self.motion = None
        self.pending_deform_p = None      # shutter-close "P" of a PointsPolygons motion block
        self.camera_motion_inv = None     # Camera::motion_inv (4x4) from a pre-World motion block
        self.mesh_p1 = {}                 # mesh index -> (n, 3) positions at shutter close
        self.env = None
        # scene contents (materials / lights / meshes / instances)
        self.meshes, self.instances, self.materials, self.lights = [], [], [], []
        self.mesh_st = {}                 # mesh index -> (n, 2) st
        self.quadrics = []                # (kind, params, material, object_to_world 3x4)
        self.patterns = []                # Scene pattern node dicts
        self.pattern_handles = {}         # handle -> node index
        self.bindings = []                # (material, field id, node)
        self.textures = []                # (H, W, 3) f32 linear RGB
        self.ies = {}                     # light index -> (v, h, candela, world_to_local)
        self.texture_ids = {}             # file path -> texture index (-1: unreadable)
        self.media = []                   # Scene medium dicts
        self.atmosphere = -1              # index into media, -1 for none
        self.curve_sets = []              # (p0, p1, v0, v1, material, object_to_world 4x4)

    # -- helpers ------------------------------------------------------------------
    def warn(self, msg):
        if msg not in self.warned:
            self.warned.append(msg)

    @property
    def ctm(self):
        return self.xf[-1]

    def apply(self, m):
        self.xf[-1] = self.xf[-1] @ m

    def object_id(self):
        name = self.state.identifier or f"object_{self.next_id}"
        if name in self.object_ids:
            return self.object_ids[name]
        i = self.next_id
        self.next_id += 1
        self.object_ids[name] = i
        return i

    def make_material(self):
        """SceneBuilder::make_material (scene_builder.rs:1850-1877)."""
        st = self.state
        if st.hair is not None:
            # A plain brown matte off curves, Marschner hair on them.
            m = marschner_hair(**st.hair)
            m["id"] = self.object_id()
            m["interior"] = st.interior
            return m
        if st.bxdf is not None:
            m = dict(st.bxdf)
        elif st.surface == "plastic":
            m = _pbr_plastic(st.color, st.roughness)
        elif st.surface == "metal":
            m = _pbr_metal(st.color, st.roughness)
        else:
            m = _pbr_matte(st.color)
        m["id"] = self.object_id()
        m["interior"] = st.interior
        if st.bxdf is not None and st.bxdf_bindings:
            m["_bindings"] = list(st.bxdf_bindings)
        return m

    def add_material(self, m):
        m = dict(m)
        for field, node in m.pop("_bindings", ()):
            self.bindings.append((len(self.materials), field, node))
        self.materials.append(m)
        return len(self.materials) - 1

    def add_light(self, type_, intensity, color, p=(0, 0, 0), e1=(0, 0, 0), e2=(0, 0, 0), radius=0.0):
        self.lights.append(dict(type=type_, intensity=float(intensity), color=tuple(color), p=tuple(p),
                                e1=tuple(e1), e2=tuple(e2), radius=float(radius)))
        return len(self.lights) - 1

    def add_mesh(self, P, I, N=None, st=None):
        self.meshes.append((np.asarray(P, np.float32).reshape(-1, 3), np.asarray(I, np.uint32).reshape(-1, 3),
                            None if N is None else np.asarray(N, np.float32).reshape(-1, 3)))
        if st is not None:
            self.mesh_st[len(self.meshes) - 1] = np.asarray(st, np.float32).reshape(-1, 2)
        return len(self.meshes) - 1

    def place(self, mesh, mat, xf, moving=True):
        """An instance of `mesh`; with `moving`, at the open MotionBegin
        block's endpoints (the reference's legacy objects, Polygon and the
        light geometry, stay put)."""
        xf1 = self.motion_endpoint(xf) if moving else None
        self.instances.append((mesh, mat, np.asarray(xf, np.float64)[:3, :].reshape(12),
                               None if xf1 is None else xf1[:3, :].reshape(12)))

    def motion_endpoint(self, current):
        """motion_endpoint (scene_builder.rs:1684-1691): the shutter-close
        transform of geometry placed at `current`: the block's T1 with the
        transforms composed after the block."""
        t0, t1 = self.state.motion_t0, self.state.motion_t1
        if t0 is None or t1 is None:
            return None
        try:
            post = np.linalg.inv(t0) @ current
        except np.linalg.LinAlgError:
            return None
        return t1 @ post

    def finish_motion_block(self, block):
        """finish_motion_block (scene_builder.rs:1637-1682): a block of
        transforms records the shutter-open and -close transforms (the
        current transform stays the open one); a block of PointsPolygons
        samples makes a deforming mesh (the last sample's "P" at shutter
        close); anything else uses its first sample."""
        name0 = block[0][0]
        if all(n in ("Translate", "Rotate", "Scale", "ConcatTransform", "Transform", "Identity") for n, _ in block):
            base = self.ctm.copy()
            self.process(*block[0])
            t0 = self.ctm.copy()
            if len(block) > 1:
                self.xf[-1] = base
                self.process(*block[-1])
                t1 = self.ctm.copy()
                self.xf[-1] = t0
                self.state.motion_t0, self.state.motion_t1 = t0, t1
            return
        if all(n == name0 for n, _ in block) and name0 in ("PointsPolygons", "PointsGeneralPolygons"):
            if len(block) > 1:
                self.pending_deform_p = _Params(block[-1][1], 2).numbers("P")
            self.process(*block[0])
            self.pending_deform_p = None
            return
        self.warn(f'MotionBegin over "{name0}" not supported (transforms and PointsPolygons deformation only); '
                  "using the first sample")
        self.process(*block[0])

    def add_quadric(self, kind, params, mat, xf):
        self.quadrics.append((kind, [float(v) for v in params], mat, np.asarray(xf, np.float64)[:3, :].reshape(12)))

    def tessellated_mesh(self, P, I, N=None, emissive=True, st=None, displace=False, P1=None):
        """add_tessellated_mesh (scene_builder.rs:1195-1234): the state's
        displacement on meshes the reference tessellates (`displace`; not
        on the quadrics it intersects analytically); quadrics take the
        plain state material (no area-light emission, :813-909). `P1`: the
        positions at shutter close of a deforming mesh (displacement
        rebuilds the mesh without them, as displace_mesh does)."""
        if displace and self.state.displace is not None:
            from .displace import displace_mesh
            P, N = displace_mesh(P, I, N, **self.state.displace)
            P1 = None
        mesh = self.add_mesh(P, I, N, st)
        if P1 is not None:
            self.mesh_p1[mesh] = np.asarray(P1, np.float32).reshape(-1, 3)
        m = self.make_material()
        if emissive and self.state.area_light is not None:
            inten, col = self.state.area_light
            m["emission"] = tuple(c * inten for c in col)
        mat = self.add_material(m)
        if self.defining is not None:
            self.defining[1].append((mesh, self.ctm.copy(), mat))
        else:
            self.place(mesh, mat, self.ctm)

    # -- requests -------------------------------------------------------------------
    def run(self, reqs):
        for name, vals in reqs:
            if self.recording is not None:
                if name == "ArchiveEnd":
                    self.archives[self.recording[0]] = self.recording[1]
                    self.recording = None
                else:
                    self.recording[1].append((name, vals))
                continue
            if self.motion is not None and name != "MotionEnd":
                self.motion.append((name, vals))
                continue
            self.process(name, vals)

    def process(self, name, vals):
        st = self.state
        if name == "WorldBegin" and st.motion_t0 is not None and st.motion_t1 is not None:
            # A motion block over the pre-World transforms animates the
            # camera (scene_builder.rs:271-285): rays use the inverse of the
            # delta t1 t0^-1; the motion state does not reach world geometry.
            try:
                self.camera_motion_inv = np.linalg.inv(st.motion_t1 @ np.linalg.inv(st.motion_t0))
            except np.linalg.LinAlgError:
                pass
            st.motion_t0 = st.motion_t1 = None
        if name in ("version", "WorldEnd", "FrameBegin", "FrameEnd", "WorldBegin", "IfBegin", "ElseIf", "Else",
                    "IfEnd", "Display", "Clipping", "ClippingPlane", "CropWindow", "FrameAspectRatio",
                    "PixelVariance", "Exposure", "Quantize", "Hider", "Integrator", "TextureCoordinates",
                    "ShadingInterpolation", "RelativeDetail", "Declare", "Orientation", "ReverseOrientation",
                    "Sides", "Opacity", "CoordinateSystem", "ScopedCoordinateSystem",
                    "Shutter", "ArchiveEnd"):
            return
        if name == "Basis":
            # Basis <name | 16 numbers> ustep <name | 16 numbers> vstep (scene_builder.rs:576-601).
            for k, attr in ((0, "basis_u"), (2, "basis_v")):
                if k < len(vals):
                    b = vals[k]
                    step = _num(vals, k + 1)
                    if isinstance(b, str) or (isinstance(b, list) and len(b) == 16):
                        setattr(st, attr, (b, step))
            return
        if name == "ShadingRate":
            r = _num(vals, 0)
            if r is not None:
                st.shading_rate = r
            return
        if name == "AttributeBegin":
            self.attr_stack.append(st.copy())
            self.xf.append(self.ctm.copy())
        elif name == "AttributeEnd":
            if self.attr_stack:
                self.state = self.attr_stack.pop()
            if len(self.xf) > 1:
                self.xf.pop()
        elif name == "TransformBegin":
            self.xf.append(self.ctm.copy())
        elif name == "TransformEnd":
            if len(self.xf) > 1:
                self.xf.pop()
        elif name == "MotionBegin":
            self.motion = []
        elif name == "MotionEnd":
            block, self.motion = self.motion or [], None
            if block:
                self.finish_motion_block(block)
        elif name == "ArchiveBegin":
            self.recording = (_str(vals, 0) or "", [])
        elif name == "ReadArchive":
            self.read_archive(_str(vals, 0))
        elif name == "ObjectBegin":
            h = _str(vals, 0) or (str(_num(vals, 0)) if _num(vals, 0) is not None else "0")
            self.attr_stack.append(st.copy())
            self.xf.append(np.eye(4))
            self.defining = (h, [])
        elif name == "ObjectEnd":
            if self.defining is not None:
                self.object_defs[self.defining[0]] = self.defining[1]
                self.defining = None
            if self.attr_stack:
                self.state = self.attr_stack.pop()
            if len(self.xf) > 1:
                self.xf.pop()
        elif name == "ObjectInstance":
            h = _str(vals, 0) or (str(_num(vals, 0)) if _num(vals, 0) is not None else "0")
            entries = self.object_defs.get(h)
            if entries is None:
                self.warn(f'ObjectInstance "{h}" has no definition')
            else:
                for mesh, local, mat in entries:
                    self.place(mesh, mat, self.ctm @ local)
        elif name == "Format":
            w, h = _num(vals, 0), _num(vals, 1)
            if w is not None and h is not None:
                self.width, self.height = int(w), int(h)
        elif name == "Projection":
            kind = _str(vals, 0)
            if kind == "perspective":
                self.projection = abi.PROJECTION_PERSPECTIVE
                fov = _Params(vals, 1).number("fov")
                if fov is not None:
                    self.fov = fov
            elif kind == "orthographic":
                self.projection = abi.PROJECTION_ORTHOGRAPHIC
            elif kind is not None:
                self.warn(f'Projection "{kind}" not implemented; using perspective')
        elif name == "DepthOfField":
            a = [_num(vals, k) for k in range(3)]
            if all(x is not None for x in a):
                self.dof = tuple(a)
        elif name == "PixelFilter":
            f = _str(vals, 0)
            if f is not None:
                xw = _num(vals, 1)
                xw = 2.0 if xw is None else xw
                yw = _num(vals, 2)
                yw = xw if yw is None else yw
                w = (xw + yw) * 0.5
                kinds = {"triangle": abi.FILTER_TRIANGLE, "gaussian": abi.FILTER_GAUSSIAN, "box": abi.FILTER_BOX}
                self.filter = (kinds[f], max(w, 1e-3)) if f in kinds else (abi.FILTER_BOX, 1.0)
        elif name == "ScreenWindow":
            # The orthographic window's half-extents (scene_builder.rs:529-534, 223-225).
            a = [_num(vals, k) for k in range(4)]
            if all(x is not None for x in a):
                self.screen_window = tuple(a)
        elif name == "PixelSamples":
            x, y = _num(vals, 0), _num(vals, 1)
            if x is not None and y is not None:
                self.pixel_samples = (max(int(x), 1), max(int(y), 1))
        elif name in ("Option", "Attribute"):
            cat = _str(vals, 0)
            p = _Params(vals, 1)
            if name == "Attribute" and cat == "identifier":
                nm = p.string("name")
                if nm is not None:
                    st.identifier = nm
            if name == "Option" and cat == "background":
                c = p.numbers("color")
                if c is not None and len(c) >= 3:
                    self.background = tuple(c[:3])
        elif name == "Identity":
            self.xf[-1] = np.eye(4)
        elif name in ("Transform", "ConcatTransform"):
            m = _as_numbers(vals[0]) if vals else None
            if m is not None and len(m) == 16:
                if name == "Transform":
                    self.xf[-1] = _from_rib(m)
                else:
                    self.apply(_from_rib(m))
        elif name == "Translate":
            a = [_num(vals, k) for k in range(3)]
            if all(x is not None for x in a):
                self.apply(_translate(*a))
        elif name == "Rotate":
            a = [_num(vals, k) for k in range(4)]
            if all(x is not None for x in a):
                self.apply(_rotate(*a))
        elif name == "Scale":
            a = [_num(vals, k) for k in range(3)]
            if all(x is not None for x in a):
                self.apply(_scale(*a))
        elif name == "Color":
            c = self.color_from(vals)
            if c is not None:
                st.color = c
        elif name == "Surface":
            s = _str(vals, 0)
            if s is not None:
                st.surface = s
                r = _Params(vals, 1).number("roughness")
                st.roughness = 0.1 if r is None else r
        elif name == "Bxdf":
            t = _str(vals, 0) or ""
            prm = _Params(vals, 2 if len(vals) % 2 == 0 else 1)
            if t == "PxrMarschnerHair":
                # HairParams::from_bxdf_params (hair.rs:82-100).
                a = prm.numbers("absorption")
                c = prm.numbers("color")
                st.hair = dict(roughness=_or(prm.number("roughness"), 0.3),
                               azimuthal_roughness=_or(prm.number("azimuthalRoughness"), 0.3),
                               ior=_or(prm.number("ior"), 1.55),
                               absorption=None if not a else (tuple(a[:3]) if len(a) >= 3 else (a[0],) * 3),
                               color=tuple(c[:3]) if c is not None and len(c) >= 3 else None)
                st.bxdf, st.bxdf_bindings = None, []
                return
            st.hair = None
            if t != "PxrSurface":
                self.warn(f'Bxdf "{t}" not implemented; treating as PxrSurface')
            st.bxdf = _pbr_bxdf(prm)
            st.bxdf_bindings = self.bxdf_bindings(prm)
        elif name == "Pattern":
            self.pattern_request(vals)
        elif name == "Curves":
            self.curves_request(vals)
        elif name == "Points":
            self.points_request(vals)
        elif name in ("Interior", "Atmosphere"):
            self.medium_request(name, vals)
        elif name == "Exterior":
            self.warn("Exterior is subsumed by nested Interior tracking (rays exiting an object return "
                      "to the enclosing medium); ignoring")
        elif name == "Displace":
            # scene_builder.rs:776-795: the built-in fBm "noise" displacement.
            kind = _str(vals, 0) or ""
            if kind != "noise":
                self.warn(f'Displace "{kind}": only the built-in "noise" displacement exists; using it')
            prm = _Params(vals, 2 if len(vals) % 2 == 0 else 1)
            d = dict(amplitude=0.1, frequency=1.0, octaves=4, gain=0.5, lacunarity=2.0, offset=(0.0, 0.0, 0.0))
            for key in ("amplitude", "frequency", "gain", "lacunarity"):
                v = prm.number(key)
                if v is not None:
                    d[key] = v
            v = prm.number("octaves")
            if v is not None:
                d["octaves"] = int(v)
            v = prm.numbers("offset")
            if v is not None and len(v) >= 3:
                d["offset"] = tuple(v[:3])
            st.displace = d
        elif name == "AreaLightSource":
            p = _Params(vals, 2 if len(vals) % 2 == 0 else 1)
            inten = p.number("intensity")
            col = p.numbers("lightcolor")
            st.area_light = (1.0 if inten is None else inten,
                             tuple(col[:3]) if col is not None and len(col) >= 3 else (1.0, 1.0, 1.0))
        elif name == "LightSource":
            self.light_source(vals)
        elif name == "Light":
            self.pxr_light(vals)
        elif name == "Polygon":
            self.polygon(vals)
        elif name in ("GeneralPolygon", "SubdivisionMesh", "HierarchicalSubdivisionMesh"):
            self.warn(f"{name} not supported; skipping")
        elif name in ("PatchMesh", "Patch"):
            self.patch_mesh(name, vals)
        elif name == "NuPatch":
            self.nu_patch(vals)
        elif name in ("PointsPolygons", "PointsGeneralPolygons"):
            self.points_polygons(name, vals)
        elif name in _QUADRIC_ARGS:
            a = [_num(vals, k) for k in range(_QUADRIC_ARGS[name])]
            if all(x is not None for x in a):
                if self.defining is not None:
                    self.warn(f"{name} inside ObjectBegin is not instanced; skipping")
                    return
                # An analytic quadric with the current transform and the
                # plain state material (scene_builder.rs:813-909).
                self.add_quadric(_QUADRIC_KIND[name], a, self.add_material(self.make_material()), self.ctm)
        elif name == "Procedural" and _str(vals, 0) == "DelayedReadArchive":
            # Loaded at once, as the reference does (scene_builder.rs:384-399).
            args = vals[1] if len(vals) > 1 else None
            f = args[0] if isinstance(args, list) and args and isinstance(args[0], str) else (
                args if isinstance(args, str) else None)
            self.warn('Procedural "DelayedReadArchive" loads eagerly (no lazy loading)')
            self.read_archive(f)
        else:
            self.warn(f"RIB request '{name}' not rendered on this path; skipping")

    def curves_request(self, vals):
        """curves_request (scene_builder.rs:1050-1119): Curves "cubic" |
        "linear" [nvertices] "nonperiodic" "P" [...] with "width" (root to
        tip) or "constantwidth"; cubic curves by the v Basis, diced into
        clamp(8 / shading rate, 2, 24) segments per span."""
        if self.defining is not None:
            self.warn("Curves inside ObjectBegin is not instanced; skipping")
            return
        kind = _str(vals, 0) or "cubic"
        nverts = _as_numbers(vals[1]) if len(vals) > 1 else None
        if nverts is None:
            self.warn("Curves without [nvertices]; skipping")
            return
        if (_str(vals, 2) or "nonperiodic") == "periodic":
            self.warn('Curves "periodic" not supported; treating as nonperiodic')
        prm = _Params(vals, 3)
        P = prm.numbers("P")
        if P is None:
            self.warn('Curves without "P"; skipping')
            return
        w = prm.numbers("width")
        if w:
            w_root, w_tip = w[0], w[-1]
        else:
            w_root = w_tip = _or(prm.number("constantwidth"), 0.01)
        cubic = None
        if kind != "linear":
            cubic = self._basis(self.state.basis_v)
        segs = min(max(int(8.0 / max(self.state.shading_rate, 0.1)), 2), 24)
        P = np.asarray(P, np.float64)
        parts, cursor = [], 0
        for nv in nverts:
            nv = int(nv)
            if (cursor + nv) * 3 > len(P):
                break
            parts.append(dice_curve(P[3 * cursor:3 * (cursor + nv)].reshape(-1, 3), cubic, w_root, w_tip, segs))
            cursor += nv
        parts = [q for q in parts if q is not None]
        if parts:
            self.add_curve_set(*(np.concatenate([q[k] for q in parts]) for k in range(4)))

    def points_request(self, vals):
        """points_request (scene_builder.rs:1122-1154): particles as
        zero-length segments (spheres) of diameter "width" (per point) or
        "constantwidth" (0.05)."""
        if self.defining is not None:
            self.warn("Points inside ObjectBegin is not instanced; skipping")
            return
        prm = _Params(vals, 0)
        P = prm.numbers("P")
        if P is None:
            self.warn('Points without "P"; skipping')
            return
        P = np.asarray(P, np.float64).reshape(-1, 3)
        widths = prm.numbers("width")
        cw = _or(prm.number("constantwidth"), 0.05)
        w = np.array([widths[i] if widths is not None and i < len(widths) else cw for i in range(len(P))])
        e = np.concatenate([P, (w * 0.5)[:, None]], axis=1)
        half = np.full(len(P), 0.5)
        self.add_curve_set(e, e, half, half)

    def add_curve_set(self, p0, p1, v0, v1):
        """add_curve_set (scene_builder.rs:1157-1170): the state material and
        the current placement."""
        mat = self.add_material(self.make_material())
        self.curve_sets.append((p0, p1, v0, v1, mat, self.ctm.copy(), self.motion_endpoint(self.ctm)))

    def medium_request(self, name, vals):
        """Interior / Atmosphere (scene_builder.rs:324-373): sigma_a, sigma_s,
        g, emission, maxdistance, and density "fbm" with frequency, octaves,
        gain, lacunarity, coverage and sharpness. Atmospheres are slabs of
        1200 units by default."""
        p = _Params(vals, 1)

        def get3(key, default):
            v = p.numbers(key)
            return tuple(v[:3]) if v is not None and len(v) >= 3 else default

        dens = p.string("density")
        fbm = None
        if dens in ("fbm", "noise"):
            fbm = {}
            for key, default in (("frequency", 0.3), ("octaves", 5.0), ("gain", 0.55), ("lacunarity", 2.0),
                                 ("coverage", 0.5), ("sharpness", 4.0)):
                v = p.number(key)
                fbm[key] = default if v is None else v
        elif dens is not None:
            self.warn(f'Interior density "{dens}" not implemented; homogeneous')
        ext = p.number("maxdistance")
        med = medium(get3("sigma_a", (0.1, 0.1, 0.1)), get3("sigma_s", (0.5, 0.5, 0.5)),
                     g=p.number("g") or 0.0, emission=get3("emission", (0.0, 0.0, 0.0)),
                     max_distance=(1200.0 if name == "Atmosphere" else math.inf) if ext is None else ext, fbm=fbm)
        self.media.append(med)
        if name == "Atmosphere":
            self.atmosphere = len(self.media) - 1
        else:
            self.state.interior = len(self.media) - 1

    def color_from(self, vals):
        a = [_num(vals, k) for k in range(3)]
        if all(x is not None for x in a):
            return tuple(a)
        v = _as_numbers(vals[0]) if vals else None
        return tuple(v[:3]) if v is not None and len(v) >= 3 else None

    def read_archive(self, name):
        """read_archive (scene_builder.rs:1448-1476): inline archives first,
        then a file beside the scene; a missing or unparsable file warns."""
        if name is None:
            return
        if self.archive_depth >= MAX_ARCHIVE_DEPTH:
            self.warn(f'ReadArchive "{name}": max depth exceeded; skipping')
            return
        if name in self.archives:
            reqs = self.archives[name]
        else:
            path = name if os.path.isabs(name) or self.base_dir is None else os.path.join(self.base_dir, name)
            try:
                reqs = parse_rib(_read_text(path))
            except OSError as e:
                self.warn(f'ReadArchive "{name}": {e.strerror}')
                return
            except RibError as e:
                self.warn(f'ReadArchive "{name}": parse error: {e}')
                return
        self.archive_depth += 1
        try:
            self.run(reqs)
        finally:
            self.archive_depth -= 1

    def polygon(self, vals):
        """Polygon (scene_builder.rs:911-950): a fan of triangles; with an
        area light on the state, a quad is also a sampleable rect light."""
        p = _Params(vals, 0).numbers("P")
        if p is None or len(p) < 9:
            return
        if self.defining is not None:
            self.warn("Polygon inside ObjectBegin is not instanced; skipping")
            return
        nv = len(p) // 3
        P = np.array(p[:3 * nv], dtype=np.float64).reshape(nv, 3)
        m = self.make_material()
        if self.state.area_light is not None:
            inten, col = self.state.area_light
            m["emission"] = tuple(c * inten for c in col)
            if len(p) == 12:
                c0 = _xf_point(self.ctm, P[0])
                e1 = _xf_point(self.ctm, P[1]) - c0
                e2 = _xf_point(self.ctm, P[3]) - c0
                m["area_light"] = self.add_light(abi.LIGHT_RECT, inten, col, p=c0, e1=e1, e2=e2)
        mat = self.add_material(m)
        I = [(0, i, i + 1) for i in range(1, nv - 1)]
        self.place(self.add_mesh(P, I), mat, self.ctm, moving=False)

    def points_polygons(self, name, vals):
        """points_polygons (scene_builder.rs:982-1051): fan-triangulated
        polygons with optional per-vertex normals."""
        if name == "PointsGeneralPolygons":
            nl = _as_numbers(vals[0]) if vals else None
            if nl is None:
                return
            if any(int(n) != 1 for n in nl):
                self.warn("PointsGeneralPolygons holes are not supported; using outer loops only")
            vals = vals[1:]
        nverts = _as_numbers(vals[0]) if len(vals) > 0 else None
        verts = _as_numbers(vals[1]) if len(vals) > 1 else None
        if nverts is None or verts is None:
            return
        prm = _Params(vals, 2)
        p = prm.numbers("P")
        if p is None:
            self.warn(f"{name} without \"P\"; skipping")
            return
        P = np.array(p, dtype=np.float64).reshape(-1, 3)
        n = prm.numbers("N")
        N = None
        if n is not None:
            if len(n) == len(p):
                N = np.array(n, dtype=np.float64).reshape(-1, 3)
            else:
                self.warn(f"{name} \"N\" is not per-vertex; ignoring normals")
        tris, cur = [], 0
        for nv in nverts:
            nv = int(nv)
            if cur + nv > len(verts):
                break
            poly = verts[cur:cur + nv]
            for i in range(1, nv - 1):
                tris.append((int(poly[0]), int(poly[i]), int(poly[i + 1])))
            cur += nv
        if not tris:
            return
        I = np.array(tris, dtype=np.int64)
        if I.max() >= len(P):
            raise RibError(f"{name}: vertex index out of range")
        stv = prm.numbers("st")
        ST = None
        if stv is not None and len(stv) * 3 == len(p) * 2:
            ST = np.array(stv, dtype=np.float64).reshape(-1, 2)
        p1, self.pending_deform_p = self.pending_deform_p, None
        P1 = np.array(p1, dtype=np.float64).reshape(-1, 3) if p1 is not None and len(p1) == len(p) else None
        self.tessellated_mesh(P, I, N, st=ST, displace=True, P1=P1)

    # -- patterns (scene_builder.rs:703-728, 1738-1846) -------------------------------
    def _ref_target(self, prm, name):
        """The node a "reference <type> <name>" ["handle:output"] parameter
        names, or None."""
        for t, v in prm.pairs:
            w = t.split()
            if "reference" in w and w[-1] == name:
                target = v if isinstance(v, str) else (v[0] if isinstance(v, list) and v and
                                                       isinstance(v[0], str) else None)
                if target is not None:
                    return self.pattern_handles.get(target.split(":")[0])
        return None

    def pattern_input(self, prm, name, default):
        node = self._ref_target(prm, name)
        if node is not None:
            return node
        v = prm.numbers(name)
        if v is not None and len(v) >= 3:
            return tuple(v[:3])
        if v is not None and len(v) >= 1:
            return (v[0],) * 3
        return tuple(default)

    def pattern_request(self, vals):
        """pattern_request: one node of the scene's pattern graph, named by
        its handle; the file-texture nodes are not carried."""
        ptype = _str(vals, 0) or ""
        start = 2 if len(vals) % 2 == 0 else 1
        handle = _str(vals, 1) if start == 2 else None
        if handle is None:
            self.warn("Pattern without a handle; skipping")
            return
        prm = _Params(vals, start)

        def color(name, default):
            v = prm.numbers(name)
            return tuple(v[:3]) if v is not None and len(v) >= 3 else default

        def number(name, default):
            v = prm.number(name)
            return default if v is None else v

        if ptype in ("PxrChecker", "checker"):
            node = dict(type=abi.PATTERN_CHECKER, color_a=color("colorA", (1.0, 1.0, 1.0)),
                        color_b=color("colorB", (0.0, 0.0, 0.0)),
                        scale=(number("sScale", 8.0), number("tScale", 8.0)))
        elif ptype in ("PxrFractal", "fractal", "noise"):
            node = dict(type=abi.PATTERN_FRACTAL, frequency=number("frequency", 1.0),
                        octaves=int(number("layers", 4.0)), gain=number("gain", 0.5),
                        lacunarity=number("lacunarity", 2.0))
        elif ptype in ("PxrMix", "mix"):
            node = dict(type=abi.PATTERN_MIX, inputs=(self.pattern_input(prm, "color1", (0.0, 0.0, 0.0)),
                                                      self.pattern_input(prm, "color2", (1.0, 1.0, 1.0)),
                                                      self.pattern_input(prm, "mix", (0.0, 0.0, 0.0))))
        elif ptype in ("PxrColorCorrect", "colorCorrect"):
            node = dict(type=abi.PATTERN_COLOR_CORRECT,
                        inputs=(self.pattern_input(prm, "inputRGB", (0.5, 0.5, 0.5)),),
                        color_a=color("gain", (1.0, 1.0, 1.0)), color_b=color("offset", (0.0, 0.0, 0.0)),
                        gamma=number("gamma", 1.0), saturation=number("saturation", 1.0))
        elif ptype in ("PxrRamp", "ramp"):
            pos = prm.numbers("positions")
            pos = [0.0, 1.0] if pos is None else list(pos)
            col = prm.numbers("colors")
            col = [0.0, 0.0, 0.0, 1.0, 1.0, 1.0] if col is None else list(col)
            n = min(len(pos), len(col) // 3)
            if n != len(pos) or n * 3 != len(col):
                self.warn(f'Pattern "{handle}": ramp positions and colours differ in count; using {n}')
            node = dict(type=abi.PATTERN_RAMP,
                        ramp=(np.array(pos[:n], np.float64), np.array(col[:3 * n], np.float64).reshape(-1, 3)),
                        use_t=prm.string("axis") == "t")
        elif ptype in ("PxrTexture", "texture", "triplanar"):
            tex = self.open_texture(prm.string("filename") or "")
            node = dict(type=abi.PATTERN_TEXTURE if ptype != "triplanar" else abi.PATTERN_TRIPLANAR,
                        texture=tex if isinstance(tex, int) else -1,
                        wrap=abi.WRAP_MODES.get(prm.string("wrapMode") or "periodic", abi.WRAP_PERIODIC))
            if isinstance(tex, dict):
                node["udim"] = tex
            if ptype == "triplanar":
                node["frequency"] = number("frequency", 1.0)
            else:
                node["scale"] = (number("scaleS", 1.0), number("scaleT", 1.0))
        else:
            self.warn(f'Pattern "{ptype}" not implemented; skipping')
            return
        self.pattern_handles[handle] = len(self.patterns)
        self.patterns.append(node)

    def open_texture(self, name):
        """open_texture (scene_builder.rs:1703-1736): a texture file (beside
        the scene) as a texture index, one that cannot be read as -1
        (magenta); a name holding <UDIM> as {tile: index} over the tiles
        1001..1100 that exist (-1 when none do)."""
        if not name:
            self.warn("Pattern texture without \"filename\"; rendering magenta")
            return -1
        if "<UDIM>" in name:
            tiles = {}
            for tile in range(1001, 1101):
                f = name.replace("<UDIM>", str(tile))
                path = f if os.path.isabs(f) or self.base_dir is None else os.path.join(self.base_dir, f)
                if os.path.exists(path):
                    idx = self.open_texture(f)
                    if idx >= 0:
                        tiles[tile] = idx
            if not tiles:
                self.warn(f'no UDIM tiles found for "{name}"')
                return -1
            return tiles
        path = name if os.path.isabs(name) or self.base_dir is None else os.path.join(self.base_dir, name)
        if path not in self.texture_ids:
            from .textures import TextureError, load_texture
            try:
                self.textures.append(load_texture(path))
                self.texture_ids[path] = len(self.textures) - 1
            except (OSError, TextureError, ValueError) as e:
                self.warn(f"texture {name}: {e}; rendering magenta")
                self.texture_ids[path] = -1
        return self.texture_ids[path]

    def bxdf_bindings(self, prm):
        """The Bxdf's "reference <type> <param>" ["handle:output"]
        connections as (field id, node) pairs."""
        out = []
        for t, v in prm.pairs:
            w = t.split()
            if "reference" not in w:
                continue
            param = w[-1]
            field = abi.PATTERN_FIELDS.get(param)
            if field is None:
                self.warn(f'reference to unsupported Bxdf param "{param}"; ignoring')
                continue
            node = self._ref_target(prm, param)
            if node is None:
                target = v if isinstance(v, str) else (v[0] if isinstance(v, list) and v else "")
                self.warn(f'Bxdf references unknown Pattern "{str(target).split(":")[0]}"; ignoring')
                continue
            out.append((field, node))
        return out

    def _basis(self, spec):
        from .patches import BASES
        b, step = spec
        if isinstance(b, str):
            if b not in BASES:
                return None
            m, default = BASES[b]
            return m, int(step) if step is not None else default
        return np.array(b, np.float64).reshape(4, 4), int(step) if step is not None else 1

    def patch_mesh(self, name, vals):
        """patch_mesh (scene_builder.rs:1324-1362): PatchMesh "type" nu
        uwrap nv vwrap params / Patch "type" params, bilinear or bicubic
        with the current Basis, diced by the shading rate."""
        from .patches import dice_segments, tessellate_bicubic, tessellate_bilinear
        ptype = _str(vals, 0)
        if ptype is None:
            return
        if name == "Patch":
            n = 2 if ptype == "bilinear" else 4
            nu, uw, nv, vw, start = n, False, n, False, 1
        else:
            nu, nv = _num(vals, 1), _num(vals, 3)
            if nu is None or nv is None:
                return
            nu, nv, uw, vw, start = int(nu), int(nv), _str(vals, 2) == "periodic", _str(vals, 4) == "periodic", 5
        p = _Params(vals, start).numbers("P")
        if p is None:
            self.warn(f'{name} without "P"; skipping')
            return
        segs = dice_segments(self.state.shading_rate)
        if ptype == "bilinear":
            mesh = tessellate_bilinear(p, nu, nv, uw, vw, segs)
        elif ptype == "bicubic":
            bu, bv = self._basis(self.state.basis_u), self._basis(self.state.basis_v)
            mesh = None if bu is None or bv is None else tessellate_bicubic(p, nu, nv, uw, vw, bu, bv, segs)
        else:
            self.warn(f'{name} type "{ptype}" not supported')
            return
        if mesh is None:
            self.warn(f"{name}: invalid control grid; skipping")
            return
        pos, idx, nrm, st = mesh
        self.tessellated_mesh(pos, idx, nrm, st=st, displace=True)

    def nu_patch(self, vals):
        """nu_patch (scene_builder.rs:1364-1411): NuPatch nu uorder [uknot]
        umin umax nv vorder [vknot] vmin vmax "P" | "Pw"; untrimmed."""
        from .patches import dice_segments, tessellate_nurbs
        nums = [_num(vals, k) for k in (0, 1, 3, 4, 5, 6, 8, 9)]
        knots = [_as_numbers(vals[k]) if k < len(vals) else None for k in (2, 7)]
        if any(v is None for v in nums) or any(k is None for k in knots):
            return
        nu, uorder, umin, umax, nv, vorder, vmin, vmax = nums
        prm = _Params(vals, 10)
        pw, p = prm.numbers("Pw"), prm.numbers("P")
        if pw is None and p is None:
            self.warn('NuPatch without "P"/"Pw"; skipping')
            return
        if prm.get("trimcurve") is not None:
            self.warn("NuPatch trim curves not supported yet; rendering untrimmed")
        base = dice_segments(self.state.shading_rate)
        nu, nv, uorder, vorder = int(nu), int(nv), int(uorder), int(vorder)
        segs_u = min(max(base * (max(nu - uorder, 0) + 1), 4), 128)
        segs_v = min(max(base * (max(nv - vorder, 0) + 1), 4), 128)
        mesh = tessellate_nurbs(nu, uorder, knots[0], umin, umax, nv, vorder, knots[1], vmin, vmax,
                                pw if pw is not None else p, pw is not None, segs_u, segs_v)
        if mesh is None:
            self.warn("NuPatch: invalid control data; skipping")
            return
        pos, idx, nrm, st = mesh
        self.tessellated_mesh(pos, idx, nrm, st=st, displace=True)

    def light_source(self, vals):
        """parse_light (scene_builder.rs:1582-1635): positions untransformed."""
        t = _str(vals, 0)
        p = _Params(vals, 2 if len(vals) % 2 == 0 else 1)
        inten = p.number("intensity")
        inten = 1.0 if inten is None else inten
        if t == "pointlight":
            f = p.numbers("from")
            pos = tuple(f[:3]) if f is not None and len(f) >= 3 else (0.0, 0.0, 0.0)
            li = self.add_light(abi.LIGHT_POINT, inten, (1.0, 1.0, 1.0), p=pos)
            f = p.string("iesProfile")
            if f is not None:
                # scene_builder.rs:1599-1614: oriented by the inverse of the
                # current transform; an unreadable file leaves it isotropic.
                from .ies import IesError, load_ies
                path = f if os.path.isabs(f) or self.base_dir is None else os.path.join(self.base_dir, f)
                try:
                    prof = load_ies(path)
                    self.ies[li] = prof + (np.linalg.inv(self.ctm)[:3, :3],)
                except (OSError, IesError, np.linalg.LinAlgError) as e:
                    self.warn(f"iesProfile {f}: {e}")
        elif t == "distantlight":
            f, to = p.numbers("from"), p.numbers("to")
            f = np.array(f[:3]) if f is not None and len(f) >= 3 else np.array([0.0, 0.0, -10.0])
            to = np.array(to[:3]) if to is not None and len(to) >= 3 else np.zeros(3)
            d = to - f
            ln = np.linalg.norm(d)
            d = d / ln if ln > 1e-6 else d
            self.add_light(abi.LIGHT_DISTANT, inten, (1.0, 1.0, 1.0), e1=d)
        elif t is not None:
            self.warn(f'LightSource "{t}" not rendered on this path; skipping')

    def pxr_light(self, vals):
        """build_light (scene_builder.rs:1488-1580)."""
        t = _str(vals, 0)
        if t is None:
            return
        p = _Params(vals, 2 if len(vals) % 2 == 0 else 1)
        inten = p.number("intensity")
        inten = 1.0 if inten is None else inten
        exposure = p.number("exposure") or 0.0
        scale = inten * 2.0 ** exposure
        col = p.numbers("lightColor")
        col = tuple(col[:3]) if col is not None and len(col) >= 3 else (1.0, 1.0, 1.0)
        xf = self.ctm
        origin = _xf_point(xf, (0, 0, 0))

        def emitter_mat(li):
            return self.add_material(emitter(tuple(c * scale for c in col), area_light=li))

        if t == "PxrRectLight":
            corner = _xf_point(xf, (-0.5, -0.5, 0))
            li = self.add_light(abi.LIGHT_RECT, scale, col, p=corner, e1=_xf_vec(xf, (1, 0, 0)),
                                e2=_xf_vec(xf, (0, 1, 0)))
            P = np.array([[-0.5, -0.5, 0], [0.5, -0.5, 0], [0.5, 0.5, 0], [-0.5, 0.5, 0]])
            self.place(self.add_mesh(P, [(0, 1, 2), (0, 2, 3)]), emitter_mat(li), xf, moving=False)
        elif t == "PxrSphereLight":
            radius = float(np.linalg.norm(_xf_vec(xf, (0.5, 0, 0))))
            li = self.add_light(abi.LIGHT_SPHERE, scale, col, p=origin, radius=radius)
            self.add_quadric(abi.QUADRIC_SPHERE, (0.5, -0.5, 0.5, 360.0), emitter_mat(li), xf)
        elif t == "PxrDiskLight":
            li = self.add_light(abi.LIGHT_DISK, scale, col, p=origin, e1=_xf_vec(xf, (0.5, 0, 0)),
                                e2=_xf_vec(xf, (0, 0.5, 0)))
            self.add_quadric(abi.QUADRIC_DISK, (0.0, 0.5, 360.0), emitter_mat(li), xf)
        elif t == "PxrDistantLight":
            d = _xf_vec(xf, (0, 0, -1))
            ln = np.linalg.norm(d)
            d = d / ln if ln > 1e-6 else d
            ang = p.number("angleExtent")
            ang = 0.53 if ang is None else ang
            self.add_light(abi.LIGHT_DISTANT, scale, col, e1=d, radius=math.radians(ang * 0.5))
        elif t == "PxrDomeLight":
            li = self.add_light(abi.LIGHT_DOME, scale, col)
            f = p.string("lightColorMap")
            if f is not None:
                path = f if os.path.isabs(f) or self.base_dir is None else os.path.join(self.base_dir, f)
                try:
                    from .envmap import read_hdr
                    if self.env is None:
                        self.env = (li, read_hdr(path))
                    else:
                        self.warn("only one environment map per scene; later PxrDomeLight maps are constant")
                except (OSError, ValueError) as e:
                    self.warn(f"PxrDomeLight map: {e}; using a constant dome")
        else:
            self.warn(f'Light "{t}" not implemented; skipping')

    def scene(self):
        s = RibScene(self.width, self.height, self.fov)
        for k, (P, I, N) in enumerate(self.meshes):
            s.add_mesh(P, I, N, st=self.mesh_st.get(k), positions1=self.mesh_p1.get(k))
        s.patterns = [dict(n) for n in self.patterns]
        s.bindings = list(self.bindings)
        s.textures = list(self.textures)
        s.ies = dict(self.ies)
        for m in self.materials:
            s.add_material(m)
        for l in self.lights:
            s._light(l["type"], l["intensity"], l["color"], p=l["p"], e1=l["e1"], e2=l["e2"], radius=l["radius"])
        if self.instances:
            s.add_instances([i[0] for i in self.instances], [i[1] for i in self.instances],
                            np.stack([i[2] for i in self.instances]))
            for k, inst in enumerate(self.instances):
                if inst[3] is not None:
                    s.instance_motion[k] = np.asarray(inst[3], np.float64)
        for kind, params, mat, xf in self.quadrics:
            s.add_quadric(kind, params, mat, xf)
        for p0, p1, v0, v1, mat, xf, xf1 in self.curve_sets:
            s.add_instance(s.add_curves(p0, p1, v0, v1), mat, np.asarray(xf, np.float64)[:3, :].reshape(12),
                           None if xf1 is None else np.asarray(xf1, np.float64)[:3, :].reshape(12))
        if self.camera_motion_inv is not None:
            s.camera_motion_inv = np.asarray(self.camera_motion_inv, np.float64)[:3, :].reshape(12)
        for med in self.media:
            s.add_medium(med)
        s.atmosphere = self.atmosphere
        s.filter, s.filter_width = self.filter
        s.projection = self.projection
        if self.screen_window is not None:
            l, r, b, t = self.screen_window
            s.ortho_half = (abs(r - l) * 0.5, abs(t - b) * 0.5)
        if self.dof is not None:
            fstop, flen, fdist = self.dof
            if math.isfinite(fstop) and fstop > 0:
                s.lens_radius, s.focal_distance = flen / (2.0 * fstop), fdist
        s.background = self.background
        if self.env is not None:
            s.env = (self.env[0], np.ascontiguousarray(self.env[1], dtype=np.float32))
        s.pixel_samples = self.pixel_samples
        s.warnings = list(self.warned)
        return s


def load_rib_string(text, base_dir=None):
    """A RibScene from RIB text (ReadArchive paths resolve against base_dir)."""
    b = _Builder(base_dir)
    b.run(parse_rib(text))
    return b.scene()


def _read_text(path):
    """A RIB file's text, decoding binary RIB (parse_rib_bytes)."""
    with open(path, "rb") as f:
        data = f.read()
    return decode_binary(data) if looks_binary(data) else data.decode("utf-8", errors="replace")


def load_rib(path):
    """A RibScene from a RIB file, text or binary (SceneBuilder::with_base_dir(dir of path))."""
    return load_rib_string(_read_text(path), os.path.dirname(os.path.abspath(path)))
