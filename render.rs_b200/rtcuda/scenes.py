"""Seeded synthetic scenes for the five workloads the path tracer is measured on.

Each generator is the specification of its scene: it builds the geometry,
materials, lights and camera directly (no RIB parsing). Sizes can be scaled
down for tests; the defaults are the full workloads.

  cornell_box            closed 2x2x2 box, two rotated boxes, ceiling light, 256^2/16 spp/depth 8
  triangle_cloud         1,000,000 jittered triangles in the unit cube + a 4,194,304-ray set,
                         1920x1080/16 spp, diffuse 0.5, one distant light
  instanced_materials    1,000 instances of 4 meshes, GGX / Oren-Nayar / rough glass, 64 point lights
  two_rooms              two 4x3x3 rooms joined by a 0.2x2.0 opening, light in the unseen room
  forest                 20 trees x ~45k triangles, 772,000 instances on a 512x512 fBm terrain,
                         1,200 point lights
"""
import numpy as np

from .scene import (Scene, affine, emitter, ggx_conductor, ggx_floor, matte, rot_y,
                    rough_dielectric)


# ---------------------------------------------------------------------------
# primitives
def quad(corner, e1, e2):
    c, a, b = (np.asarray(v, dtype=np.float64) for v in (corner, e1, e2))
    return np.array([c, c + a, c + a + b, c + b]), np.array([[0, 1, 2], [0, 2, 3]])


def unit_cube():
    """Axis-aligned cube [-0.5, 0.5]^3 as 12 outward-wound triangles."""
    p = np.array([[x, y, z] for z in (-0.5, 0.5) for y in (-0.5, 0.5) for x in (-0.5, 0.5)])
    faces = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    idx = []
    for a, b, c, d in faces:
        idx += [[a, b, c], [a, c, d]]
    return p, np.array(idx)


def merge(parts):
    pos, idx, off = [], [], 0
    for p, i in parts:
        pos.append(p)
        idx.append(np.asarray(i) + off)
        off += len(p)
    return np.concatenate(pos), np.concatenate(idx)


# ---------------------------------------------------------------------------
# C1: Cornell-like box
def cornell_box(width=256, height=256):
    """Closed box [-1,1]^3 open toward +z: floor, ceiling, back (0.73 grey),
    left wall (0.63, 0.065, 0.05), right wall (0.14, 0.45, 0.09) — 5 inward
    quads, 10 triangles. Two boxes (a unit cube mesh instanced twice: 0.6x1.2x0.6
    rotated 17 deg, 0.6^3 rotated -18 deg; grey Oren-Nayar sigma 0). A 0.5x0.5
    ceiling quad of radiance (17, 12, 4) that is both geometry and a rect light.
    Pinhole camera at z = +3.9 looking at the origin, 40 deg vertical fov."""
    s = Scene(width, height, fov=40.0)
    s.look_at((0.0, 0.0, 3.9), (0.0, 0.0, 0.0))
    white = s.add_material(matte((0.73, 0.73, 0.73), id=1))
    red = s.add_material(matte((0.63, 0.065, 0.05), id=2))
    green = s.add_material(matte((0.14, 0.45, 0.09), id=3))
    grey = s.add_material(matte((0.73, 0.73, 0.73), sigma=0.0, id=4))
    walls = merge([
        quad((-1, -1, 1), (2, 0, 0), (0, 0, -2)),    # floor (normal +y)
        quad((-1, 1, -1), (2, 0, 0), (0, 0, 2)),     # ceiling (normal -y)
        quad((-1, -1, -1), (2, 0, 0), (0, 2, 0)),    # back (normal +z)
    ])
    s.add_instance(s.add_mesh(*walls), white)
    s.add_instance(s.add_mesh(*quad((-1, -1, -1), (0, 2, 0), (0, 0, 2))), red)     # left, +x
    s.add_instance(s.add_mesh(*quad((1, -1, -1), (0, 0, 2), (0, 2, 0))), green)    # right, -x
    cube = s.add_mesh(*unit_cube())
    tall = affine(rot_y(17.0) @ np.diag([0.6, 1.2, 0.6]), (-0.35, -0.399, -0.3))
    short = affine(rot_y(-18.0) @ np.diag([0.6, 0.6, 0.6]), (0.35, -0.699, 0.3))
    s.add_instance(cube, grey, tall)
    s.add_instance(cube, grey, short)
    s.add_emissive_quad((-0.25, 0.999, -0.25), (0.5, 0.0, 0.0), (0.0, 0.0, 0.5), (17.0, 12.0, 4.0))
    s.materials[-1]["id"] = 5
    return s


CORNELL = dict(spp=16, max_depth=8, rr_start=3)


# ---------------------------------------------------------------------------
# C2: triangle cloud traversal stress
def triangle_cloud_mesh(n_tris=1_000_000, seed=2024):
    """Triangles with centres uniform in [-0.5, 0.5]^3 and each vertex =
    centre + N(0, 0.01^2) per axis, stored as f32 (non-indexed soup)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.5, 0.5, size=(n_tris, 1, 3))
    verts = centres + rng.normal(0.0, 0.01, size=(n_tris, 3, 3))
    pos = verts.reshape(-1, 3).astype(np.float32)
    idx = np.arange(3 * n_tris, dtype=np.uint32).reshape(-1, 3)
    return pos, idx


def triangle_cloud_rays(n_rays=4_194_304, seed=4242):
    """Ray set in the plane layout the batch API takes: (n,4) origins
    (w unused) then (n,4) directions with tmax in w. Origins are uniform on
    the radius-2 sphere, directions point at uniform points in the cube and
    are normalised; tmax = +inf."""
    rng = np.random.default_rng(seed)
    g = rng.normal(size=(n_rays, 3))
    origin = 2.0 * g / np.linalg.norm(g, axis=1, keepdims=True)
    target = rng.uniform(-0.5, 0.5, size=(n_rays, 3))
    d = target - origin
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    planes = np.zeros((2, n_rays, 4), dtype=np.float32)
    planes[0, :, :3] = origin
    planes[1, :, :3] = d
    planes[1, :, 3] = np.inf
    return planes


def triangle_cloud(width=1920, height=1080, n_tris=1_000_000, seed=2024):
    """Render form: the cloud with diffuse albedo 0.5 under one distant light."""
    s = Scene(width, height, fov=40.0)
    s.look_at((0.0, 0.0, 2.2), (0.0, 0.0, 0.0))
    mat = s.add_material(matte((0.5, 0.5, 0.5), id=1))
    s.add_instance(s.add_mesh(*triangle_cloud_mesh(n_tris, seed)), mat)
    s.add_distant_light((-0.4, -1.0, -0.3), 3.0)
    s.background = (0.1, 0.1, 0.1)
    return s


TRIANGLE_CLOUD = dict(spp=16, max_depth=8, rr_start=3)
