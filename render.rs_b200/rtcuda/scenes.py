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
  media_cornell          the Cornell box with participating media (fog, an fBm cloud in a
                         volume hull, glass with an absorbing interior) and a subsurface sphere
  furball                a sphere groomed with cubic b-spline strands of Marschner hair
"""
import numpy as np

from . import abi
from .scene import (Scene, affine, emitter, ggx_conductor, ggx_floor, marschner_hair, matte, medium, rot_y,
                    rough_dielectric, volume_hull)


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
def cornell_box(width=256, height=256, light_size=0.5, light_radiance=(17.0, 12.0, 4.0)):
    """Closed box [-1,1]^3 open toward +z: floor, ceiling, back (0.73 grey),
    left wall (0.63, 0.065, 0.05), right wall (0.14, 0.45, 0.09) — 5 inward
    quads, 10 triangles. Two boxes (a unit cube mesh instanced twice: 0.6x1.2x0.6
    rotated 17 deg, 0.6^3 rotated -18 deg; grey Oren-Nayar sigma 0). A 0.5x0.5
    ceiling quad of radiance (17, 12, 4) that is both geometry and a rect light
    (`light_size` and `light_radiance` change it). Pinhole camera at z = +3.9
    looking at the origin, 40 deg vertical fov."""
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
    h = 0.5 * light_size
    s.add_emissive_quad((-h, 0.999, -h), (light_size, 0.0, 0.0), (0.0, 0.0, light_size), tuple(light_radiance))
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


# ---------------------------------------------------------------------------
# C3: instanced materials
def icosphere(subdivisions=5):
    """Unit icosphere: 20 * 4^s triangles, smooth vertex normals (= positions)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    p = np.array(verts)
    return p, np.array(faces, dtype=np.uint32), p.copy()


def value_noise_fbm(x, y, rng_seed, octaves=5, base=4.0):
    """Seeded fBm of bilinear-smoothstep value noise on a lattice (sum of
    octaves with frequency x2 and amplitude x0.5)."""
    rng = np.random.default_rng(rng_seed)
    out = np.zeros_like(x)
    amp, freq = 1.0, base
    for _ in range(octaves):
        n = int(np.ceil(freq)) + 2
        lat = rng.uniform(-1, 1, size=(n + 1, n + 1))
        fx, fy = x * freq, y * freq
        ix, iy = np.floor(fx).astype(int), np.floor(fy).astype(int)
        tx, ty = fx - ix, fy - iy
        sx, sy = tx * tx * (3 - 2 * tx), ty * ty * (3 - 2 * ty)
        ix, iy = np.clip(ix, 0, n - 1), np.clip(iy, 0, n - 1)
        a = lat[ix, iy] * (1 - sx) + lat[ix + 1, iy] * sx
        b = lat[ix, iy + 1] * (1 - sx) + lat[ix + 1, iy + 1] * sx
        out += amp * (a * (1 - sy) + b * sy)
        amp *= 0.5
        freq *= 2.0
    return out


def fbm_grid(n=128, seed=0, amplitude=0.15, size=1.0):
    """n x n quads (2 n^2 triangles) over [-size/2, size/2]^2 in xz with an
    fBm height field in y."""
    u = np.linspace(0.0, 1.0, n + 1)
    X, Z = np.meshgrid(u, u, indexing="ij")
    H = value_noise_fbm(X, Z, seed) * amplitude
    pos = np.stack([(X - 0.5) * size, H, (Z - 0.5) * size], axis=-1).reshape(-1, 3)
    i = np.arange(n)
    a = (i[:, None] * (n + 1) + i[None, :]).reshape(-1)
    b, c, d = a + 1, a + n + 2, a + n + 1
    idx = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)])
    return pos, idx.astype(np.uint32)


def random_rotations(rng, n):
    """Uniform random rotations from unit quaternions."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)


def instanced_materials(width=1920, height=1080, n_instances=1000, n_lights=64, seed=7, subdivisions=5,
                        grid=128):
    """1,000 instances of 4 base meshes (an icosphere subdivided 5 times =
    20,480 triangles; three fBm-displaced 128x128 grid patches = 32,768
    triangles each) under seeded uniform rotation, uniform scale in [0.2, 1]
    and translation in a 20 x 5 x 20 box (y up). Per-instance materials: 60%
    GGX conductor (roughness U[0.05, 0.8], F0 U[0.02, 0.9]), 30% Oren-Nayar
    (sigma U[0, 0.5], albedo U[0.3, 0.9]^3), 10% rough dielectric (IOR 1.5,
    roughness 0.05). 64 point lights of log-uniform power P in [1, 100];
    a point light's intensity is P / (4 pi) so that its light-BVH power
    (luminance * 4 pi, src/scene/light_sampler.rs:54) equals P."""
    rng = np.random.default_rng(seed)
    s = Scene(width, height, fov=40.0)
    s.look_at((0.0, 9.0, -23.0), (0.0, 1.5, 0.0))
    s.background = (0.02, 0.02, 0.03)
    meshes = [s.add_mesh(*icosphere(subdivisions)[:2], normals=icosphere(subdivisions)[2])]
    for k in range(3):
        meshes.append(s.add_mesh(*fbm_grid(grid, seed=seed * 10 + k)))
    kind = rng.uniform(size=n_instances)
    for i in range(n_instances):
        if kind[i] < 0.6:
            m = ggx_conductor(rng.uniform(0.02, 0.9), rng.uniform(0.05, 0.8), id=i + 1)
        elif kind[i] < 0.9:
            m = matte(tuple(rng.uniform(0.3, 0.9, 3)), sigma=rng.uniform(0.0, 0.5), id=i + 1)
        else:
            m = rough_dielectric(1.5, 0.05, id=i + 1)
        s.add_material(m)
    mesh_ids = rng.integers(0, 4, size=n_instances)
    R = random_rotations(rng, n_instances)
    scale = rng.uniform(0.2, 1.0, size=n_instances)
    t = np.stack([rng.uniform(-10, 10, n_instances), rng.uniform(0, 5, n_instances),
                  rng.uniform(-10, 10, n_instances)], 1)
    xf = np.zeros((n_instances, 3, 4))
    xf[:, :, :3] = R * scale[:, None, None]
    xf[:, :, 3] = t
    s.add_instances(mesh_ids, np.arange(n_instances), xf.reshape(n_instances, 12))
    power = np.exp(rng.uniform(np.log(1.0), np.log(100.0), size=n_lights))
    lp = np.stack([rng.uniform(-11, 11, n_lights), rng.uniform(0.5, 7, n_lights), rng.uniform(-11, 11, n_lights)], 1)
    for k in range(n_lights):
        s.add_point_light(tuple(lp[k]), power[k] / (4 * np.pi))
    return s


INSTANCED_MATERIALS = dict(spp=64, max_depth=12, rr_start=3)


# ---------------------------------------------------------------------------
# C4: two rooms, light in the unseen one
def two_rooms(width=1280, height=720):
    """Two 4 x 3 x 3 rooms (x in [0,4] and [4,8], y up, z in [0,3]) joined by a
    partition at x = 4 with one 0.2 (z) x 2.0 (y) opening at z in [1.4, 1.6].
    A single 1 x 1 area light of radiance 50 hangs horizontally 0.4 below the
    second room's ceiling (y = 2.6, x in [6, 7], z in [1, 2]); the camera
    cannot see it, and of the first room only a small patch of its back wall
    sees it through the opening, so nearly all light in the camera's room is
    indirect. The panel emits from both faces (rect lights are double-sided),
    so it is kept well away from every surface: a panel a centimetre from a
    wall lights a thin band of that wall with near-singular NEE weights,
    whose fireflies would swamp any comparison of estimators. Walls and
    ceiling: Oren-Nayar albedo 0.7, sigma 0.3; floor: GGX-coated diffuse,
    roughness 0.3. The camera sits in the first room looking at the
    partition."""
    s = Scene(width, height, fov=60.0)
    s.look_at((0.35, 1.4, 1.2), (4.0, 1.1, 1.5))
    wall = s.add_material(matte((0.7, 0.7, 0.7), sigma=0.3, id=1))
    floor = s.add_material(ggx_floor((0.7, 0.7, 0.7), 0.3, id=2))
    walls = merge([
        quad((0, 3, 0), (8, 0, 0), (0, 0, 3)),        # ceiling
        quad((0, 0, 0), (0, 3, 0), (8, 0, 0)),        # z = 0 wall
        quad((0, 0, 3), (8, 0, 0), (0, 3, 0)),        # z = 3 wall
        quad((0, 0, 0), (0, 0, 3), (0, 3, 0)),        # x = 0 wall
        quad((8, 0, 0), (0, 3, 0), (0, 0, 3)),        # x = 8 wall
        # partition x = 4 with the opening z in [1.4, 1.6], y in [0, 2]
        quad((4, 0, 0), (0, 3, 0), (0, 0, 1.4)),
        quad((4, 0, 1.6), (0, 3, 0), (0, 0, 1.4)),
        quad((4, 2, 1.4), (0, 1, 0), (0, 0, 0.2)),
    ])
    s.add_instance(s.add_mesh(*walls), wall)
    s.add_instance(s.add_mesh(*quad((0, 0, 0), (0, 0, 3), (8, 0, 0))), floor)
    # Light panel hanging in the second room, facing down (normal = e1 x e2).
    s.add_emissive_quad((6.0, 2.6, 1.0), (1, 0, 0), (0, 0, 1), (50.0, 50.0, 50.0))
    s.materials[-1]["id"] = 3
    return s


TWO_ROOMS = dict(max_depth=16, rr_start=3)


# ---------------------------------------------------------------------------
# C5: forest
def _cylinder(p0, p1, r0, r1, sides=8):
    axis = p1 - p0
    L = np.linalg.norm(axis)
    a = axis / max(L, 1e-9)
    t = np.cross(a, [1.0, 0.0, 0.0] if abs(a[0]) < 0.9 else [0.0, 1.0, 0.0])
    t /= np.linalg.norm(t)
    b = np.cross(a, t)
    ang = np.linspace(0, 2 * np.pi, sides, endpoint=False)
    ring = np.cos(ang)[:, None] * t + np.sin(ang)[:, None] * b
    pos = np.concatenate([p0 + r0 * ring, p1 + r1 * ring])
    k = np.arange(sides)
    k1 = (k + 1) % sides
    idx = np.concatenate([np.stack([k, k1, k1 + sides], 1), np.stack([k, k1 + sides, k + sides], 1)])
    return pos, idx


def tree(seed, levels=7, children=3, leaves_per_tip=20, sides=8):
    """Seeded L-system-like tree: a trunk that branches `children` ways per
    level (random tilt and twist, tapering radius), 8-sided branch prisms,
    and `leaves_per_tip` leaf quads around every tip. Returns (bark, leaves)
    meshes; with the defaults about 17k bark + 29k leaf triangles."""
    rng = np.random.default_rng(seed)
    bark, leaves = [], []
    stack = [(np.zeros(3), np.array([0.0, 1.0, 0.0]), 4.0, 0.35, 0)]
    while stack:
        p, d, L, r, lvl = stack.pop()
        q = p + d * L
        bark.append(_cylinder(p, q, r, r * 0.7, sides))
        if lvl + 1 >= levels:
            for _ in range(leaves_per_tip):
                c = q + rng.normal(scale=0.6, size=3)
                e1 = rng.normal(size=3)
                e1 = e1 / np.linalg.norm(e1) * 0.35
                e2 = np.cross(e1, rng.normal(size=3))
                e2 = e2 / max(np.linalg.norm(e2), 1e-9) * 0.25
                leaves.append(quad(c - 0.5 * (e1 + e2), e1, e2))
            continue
        for k in range(children):
            tilt = rng.uniform(0.35, 0.8)
            phi = rng.uniform(0, 2 * np.pi) + k * 2 * np.pi / children
            t = np.cross(d, [1.0, 0.0, 0.0] if abs(d[0]) < 0.9 else [0.0, 0.0, 1.0])
            t /= np.linalg.norm(t)
            b = np.cross(d, t)
            nd = np.cos(tilt) * d + np.sin(tilt) * (np.cos(phi) * t + np.sin(phi) * b)
            nd /= np.linalg.norm(nd)
            stack.append((q, nd, L * rng.uniform(0.6, 0.8), r * 0.7, lvl + 1))
    return merge(bark), merge(leaves)


def forest(width=3840, height=2160, n_trees=20, n_placements=386_000, n_lights=1200, seed=11, terrain=512,
           tree_levels=7, extent=1000.0):
    """20 seeded trees (bark + leaf meshes, ~45k triangles per tree; leaves
    use a constant presence cutout of 0.5) placed 386,000 times with jitter on
    a 1 km^2 fBm terrain (512 x 512 grid): every placement is two instances
    (bark, leaves), 772,000 instances in all. 1,200 point lights with colour
    U[0,1]^3 and log-uniform power in [0.1, 1000] (intensity = P / 4pi)."""
    rng = np.random.default_rng(seed)
    s = Scene(width, height, fov=45.0)
    half = extent / 2
    s.background = (0.01, 0.01, 0.02)
    bark_m = s.add_material(matte((0.30, 0.20, 0.12), sigma=0.4, id=1))
    leaf_m = s.add_material(matte((0.15, 0.45, 0.12), sigma=0.2, presence=0.5, id=2))
    ground_m = s.add_material(matte((0.35, 0.30, 0.22), sigma=0.5, id=3))
    tpos, tidx = fbm_grid(terrain, seed=seed, amplitude=40.0 / extent, size=1.0)
    tpos = tpos * extent
    s.add_instance(s.add_mesh(tpos, tidx), ground_m)
    ids = []
    for k in range(n_trees):
        bark, leaves = tree(seed * 100 + k, levels=tree_levels)
        ids.append((s.add_mesh(*bark), s.add_mesh(*leaves)))
    # Jittered placements on the terrain (height looked up from the grid).
    g = int(np.ceil(np.sqrt(n_placements)))
    cell = extent / g
    k = np.arange(n_placements)
    xz = np.stack([(k % g + rng.uniform(0.1, 0.9, n_placements)) * cell - half,
                   (k // g + rng.uniform(0.1, 0.9, n_placements)) * cell - half], 1)
    hgrid = tpos[:, 1].reshape(terrain + 1, terrain + 1)
    gi = np.clip(((xz + half) / extent * terrain).astype(int), 0, terrain)
    y = hgrid[gi[:, 0], gi[:, 1]] - 0.2
    which = rng.integers(0, n_trees, n_placements)
    ang = rng.uniform(0, 2 * np.pi, n_placements)
    sc = rng.uniform(0.7, 1.3, n_placements)
    c, si = np.cos(ang) * sc, np.sin(ang) * sc
    xf = np.zeros((n_placements, 3, 4))
    xf[:, 0, 0], xf[:, 0, 2], xf[:, 1, 1], xf[:, 2, 0], xf[:, 2, 2] = c, si, sc, -si, c
    xf[:, :, 3] = np.stack([xz[:, 0], y, xz[:, 1]], 1)
    xf = xf.reshape(n_placements, 12)
    bark_ids = np.array([ids[w][0] for w in which])
    leaf_ids = np.array([ids[w][1] for w in which])
    s.add_instances(bark_ids, np.full(n_placements, bark_m), xf)
    s.add_instances(leaf_ids, np.full(n_placements, leaf_m), xf)
    power = np.exp(rng.uniform(np.log(0.1), np.log(1000.0), size=n_lights))
    col = rng.uniform(0, 1, size=(n_lights, 3))
    lx = rng.uniform(-half, half, size=(n_lights, 2))
    lgi = np.clip(((lx + half) / extent * terrain).astype(int), 0, terrain)
    ly = hgrid[lgi[:, 0], lgi[:, 1]] + rng.uniform(2.0, 12.0, n_lights)
    for j in range(n_lights):
        s.add_point_light((lx[j, 0], ly[j], lx[j, 1]), power[j] / (4 * np.pi), tuple(col[j]))
    cy = hgrid[terrain // 2, terrain // 2]
    s.look_at((0.0, cy + 35.0, -half * 0.35), (0.0, cy, 0.0))
    return s


FOREST = dict(spp=32, max_depth=10, rr_start=3)


def patterned_room(width=96, height=72):
    """A small room whose materials are driven by procedural patterns
    (src/texture/pattern.rs): a checker floor (8 x 8 cells over st, fine
    enough that the ray-cone footprint blends it far away), a back wall
    whose diffuse colour mixes a ramp over s with a colour-corrected fBm,
    fBm-driven specular roughness on a plastic block placed with a 0.5
    scale (st density doubles in world units), and a ceiling light."""
    s = Scene(width, height, fov=50.0)
    s.look_at((0.0, 1.0, -3.2), (0.0, 0.8, 0.0))
    st_quad = np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]])

    def quad_mesh(corner, e1, e2):
        p, i = quad(corner, e1, e2)
        return s.add_mesh(p, i, st=st_quad)

    checker = s.add_checker((0.8, 0.8, 0.8), (0.1, 0.1, 0.1), scale=(8.0, 8.0))
    floor_m = s.add_material(matte((1.0, 1.0, 1.0)))
    s.bind_pattern(floor_m, "diffuseColor", checker)
    s.add_instance(quad_mesh((-2, 0, -4), (0, 0, 6), (4, 0, 0)), floor_m)

    ramp = s.add_ramp([0.0, 0.5, 1.0], [[0.9, 0.2, 0.1], [0.2, 0.8, 0.2], [0.1, 0.3, 0.9]])
    noise = s.add_fractal(frequency=3.0, octaves=4, gain=0.5, lacunarity=2.0)
    graded = s.add_color_correct(noise, gain=(1.2, 1.0, 0.8), offset=(0.0, 0.05, 0.1), gamma=1.5, saturation=0.6)
    wall = s.add_mix(ramp, graded, 0.4)
    wall_m = s.add_material(matte((1.0, 1.0, 1.0)))
    s.bind_pattern(wall_m, "diffuseColor", wall)
    s.add_instance(quad_mesh((-2, 0, 2), (4, 0, 0), (0, 3, 0)), wall_m)
    side = s.add_material(matte((0.6, 0.6, 0.6)))
    s.add_instance(quad_mesh((-2, 0, -4), (0, 3, 0), (0, 0, 6)), side)
    s.add_instance(quad_mesh((2, 0, -4), (0, 0, 6), (0, 3, 0)), side)
    s.add_instance(quad_mesh((-2, 3, -4), (4, 0, 0), (0, 0, 6)), side)

    rough = s.add_fractal(frequency=6.0, octaves=3)
    block_m = s.add_material(ggx_floor((0.7, 0.5, 0.3), 0.3))
    s.bind_pattern(block_m, "specularRoughness", rough)
    s.bind_pattern(block_m, "diffuseColor", s.add_checker((0.9, 0.6, 0.2), (0.2, 0.3, 0.8), scale=(4.0, 4.0)))
    # The cube with one st square per face (unshared corners).
    cp, ci = unit_cube()
    corners = np.concatenate([cp[[t0[0], t0[1], t0[2], t1[2]]] for t0, t1 in zip(ci[0::2], ci[1::2])])
    idx = np.array([[4 * f, 4 * f + 1, 4 * f + 2, 4 * f, 4 * f + 2, 4 * f + 3] for f in range(6)]).reshape(-1, 3)
    block = s.add_mesh(corners, idx, st=np.tile(st_quad, (6, 1)))
    s.add_instance(block, block_m, affine(rot_y(25) * 0.5, (0.4, 0.5, 0.6)))

    s.add_emissive_quad((-0.5, 2.99, -0.5), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (12.0, 11.0, 9.0))
    return s


# ---------------------------------------------------------------------------
# Participating media and subsurface scattering
def media_cornell(width=64, height=64, fog=True, cloud=True, glass=True, sss=True, point_light=True):
    """The Cornell box (cornell_box) with the reference's media and
    subsurface features, each switchable:
      fog    an atmosphere of thin forward-scattering haze (sigma_s 0.12-0.16,
             sigma_a 0.01, g 0.5, 8 units deep);
      cloud  a volume-hull sphere (r 0.3, mid-air) holding an fBm cloud
             (sigma_s 4, g 0.6, frequency 2, 3 octaves, coverage 0.6);
      glass  a rough-glass sphere (r 0.25, on the floor) with an absorbing
             amber interior;
      sss    a sphere (r 0.22, on the floor) whose paths take the subsurface
             walk (gain 1, colour (0.9, 0.5, 0.3), mean free path 0.2/0.1/0.05);
      point_light  a warm point light under the ceiling (equiangular NEE).
    Scenes with media render with 64 bounces (the reference's rule)."""
    s = cornell_box(width, height)
    if point_light:
        s.add_point_light((0.45, 0.7, 0.4), 0.8, (1.0, 0.85, 0.6))
    if fog:
        s.add_medium(medium((0.01, 0.01, 0.01), (0.12, 0.14, 0.16), g=0.5, max_distance=8.0), atmosphere=True)
    sphere = [1.0, -1.0, 1.0, 360.0]
    if cloud:
        ci = s.add_medium(medium((0.05, 0.05, 0.05), (4.0, 4.0, 4.0), g=0.6,
                                 fbm=dict(frequency=2.0, octaves=3, gain=0.5, lacunarity=2.0, coverage=0.6,
                                          sharpness=3.0)))
        hull = s.add_material(volume_hull(interior=ci, id=6))
        s.add_quadric(abi.QUADRIC_SPHERE, sphere, hull, affine(np.eye(3) * 0.3, (-0.05, 0.35, 0.0)))
    if glass:
        gi = s.add_medium(medium((0.9, 0.35, 0.08), (0.0, 0.0, 0.0)))
        gm = s.add_material(rough_dielectric(1.5, 0.05, interior=gi, id=7))
        s.add_quadric(abi.QUADRIC_SPHERE, sphere, gm, affine(np.eye(3) * 0.25, (-0.55, -0.75, 0.55)))
    if sss:
        sm = s.add_material(matte((0.8, 0.8, 0.8), subsurface_gain=1.0, subsurface_color=(0.9, 0.5, 0.3),
                                  subsurface_dmfp=(0.2, 0.1, 0.05), id=8))
        s.add_quadric(abi.QUADRIC_SPHERE, sphere, sm, affine(np.eye(3) * 0.22, (0.05, -0.78, 0.7)))
    return s


# ---------------------------------------------------------------------------
# Curves and hair
def furball(width=128, height=64, n_strands=20_000, seed=5):
    """A unit sphere of skin (an analytic quadric) groomed with `n_strands`
    cubic b-spline strands of 6 control points (3 spans x 8 segments each,
    dice_curve), 0.35 long, swept sideways, 0.012 wide at the root and
    0.002 at the tip, shaded with Marschner hair (colour (0.32, 0.14,
    0.05), roughness 0.35 / 0.32); a constant blue dome and a warm rect
    key light. The layout of the reference's furball scene with a seeded
    groom of its own."""
    from .patches import BASES
    from .rib import dice_curve
    s = Scene(width, height, fov=26.0)
    s.look_at((0.0, 1.3, 0.0), (0.0, 1.3, 9.5))
    s.add_dome_light(0.6, (0.6, 0.7, 1.0))
    s.add_rect_light((-4.5, 6.0, 2.5), (3.0, 0.0, 0.0), (0.0, 0.0, 3.0), 6.0, (1.0, 0.9, 0.8))
    centre = np.array([0.0, 1.32, 9.5])
    skin = s.add_material(matte((0.30, 0.17, 0.08)))
    s.add_quadric(abi.QUADRIC_SPHERE, [1.0, -1.0, 1.0, 360.0], skin, affine(np.eye(3), centre))
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n_strands, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    side = np.cross(d, [0.3, 1.0, 0.1])
    side /= np.linalg.norm(side, axis=1, keepdims=True)
    sj = np.arange(6) / 5 * 0.35
    ctrl = (d[:, None, :] * (1.0 + sj[None, :, None]) + side[:, None, :] * (0.32 * sj * sj)[None, :, None]
            + np.array([0.0, -0.1, 0.0]) * (sj * sj)[None, :, None])
    parts = [dice_curve(c, (BASES["b-spline"][0], 1), 0.012, 0.002, 8) for c in ctrl]
    p0, p1, v0, v1 = (np.concatenate([q[k] for q in parts]) for k in range(4))
    coat = s.add_material(marschner_hair(color=(0.32, 0.14, 0.05), roughness=0.35, azimuthal_roughness=0.32))
    s.add_instance(s.add_curves(p0, p1, v0, v1), coat, affine(np.eye(3), centre))
    return s



def motion_cornell(width=64, height=64, transform=True, deform=True, camera=True):
    """The Cornell box with motion blur (src/geometry/mesh.rs:230-304,
    camera.rs:85-146): the tall box slides 0.5 toward +x and turns a further
    20 deg over the shutter (transform motion), a glossy sheet with vertex
    normals bends (its far edge rises 0.4 at shutter close: deformation, so
    its shading takes the geometric normal), and the camera drifts 0.15
    along +x (camera motion, as the inverse delta the reference stores).
    Each part can be left static."""
    s = cornell_box(width, height)
    tall = 3   # instance of the tall box (walls, left, right, tall, short, light)
    if transform:
        s.instance_motion[tall] = affine(rot_y(37.0) @ np.diag([0.6, 1.2, 0.6]), (0.15, -0.399, -0.3))
    p, i = quad((-0.2, -0.2, 0.4), (0.6, 0.0, 0.0), (0.0, 0.0, 0.5))
    p = np.asarray(p, np.float32)
    p1 = p.copy()
    p1[np.isclose(p[:, 2], 0.9), 1] += 0.4
    nrm = np.tile(np.array([[0.0, 1.0, 0.0]], np.float32), (len(p), 1))
    sheet = s.add_mesh(p, i, normals=nrm, positions1=p1 if deform else None)
    s.add_instance(sheet, s.add_material(ggx_floor((0.8, 0.7, 0.3), 0.35)))
    if camera:
        s.camera_motion_inv = affine(np.eye(3), (-0.15, 0.0, 0.0))
    return s


def pattern_cutouts(width=64, height=48):
    """Cutouts driven by patterns (a presence binding, the reference's
    texture-alpha leaves): a screen whose presence is a 6 x 6 checker of 1
    and 0 (square holes), a second one whose presence is fBm noise (graded
    partial cover), both between a ceiling light and the floor so that
    their shadows and the views through them depend on the pattern at every
    blocker."""
    s = Scene(width, height, fov=50.0)
    s.look_at((0.0, 1.2, -3.0), (0.0, 0.6, 0.0))
    st_quad = np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]])
    white = s.add_material(matte((0.75, 0.75, 0.75)))
    s.add_instance(s.add_mesh(*quad((-2, 0, -3), (0, 0, 5), (4, 0, 0))), white)
    s.add_instance(s.add_mesh(*quad((-2, 0, 2), (4, 0, 0), (0, 3, 0))), white)
    holes = s.add_material(matte((0.8, 0.3, 0.2)))
    s.bind_pattern(holes, "presence", s.add_checker((1, 1, 1), (0, 0, 0), scale=(6.0, 6.0)))
    p, i = quad((-1.2, 0.9, -0.6), (1.1, 0.0, 0.0), (0.0, 0.3, 1.2))
    s.add_instance(s.add_mesh(p, i, st=st_quad), holes)
    veil = s.add_material(ggx_floor((0.2, 0.5, 0.8), 0.3))
    s.bind_pattern(veil, "presence", s.add_fractal(frequency=4.0, octaves=3))
    p, i = quad((0.2, 0.4, -0.4), (0.9, 0.0, 0.0), (0.0, 0.9, 0.6))
    s.add_instance(s.add_mesh(p, i, st=st_quad), veil)
    s.add_rect_light((-0.6, 2.6, -0.6), (1.2, 0.0, 0.0), (0.0, 0.0, 1.2), 8.0)
    return s
