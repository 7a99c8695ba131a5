"""The BVH builder on the GPU (bvh_build.cu) against the host builder
(flatten.cpp): both follow the reference's binned-SAH rules
(src/accel/bvh.rs:256-345) and the same 8-wide collapse, so the trees must
agree node for node: equal node counts, bit-identical closest-hit distances
and hit records, and bit-identical renders. Only the order of primitives
inside a leaf may differ, which changes which of two triangles at exactly the
same distance reports the hit."""
import numpy as np
import pytest

from rtcuda import PtSession, abi, scenes
from rtcuda.scene import Scene, matte

pytestmark = pytest.mark.gpu
MISS = 0xFFFFFFFF


def _rays(n, seed, lo=-1.0, hi=1.0, radius=3.0):
    rng = np.random.default_rng(seed)
    g = rng.normal(size=(n, 3))
    o = radius * g / np.linalg.norm(g, axis=1, keepdims=True)
    d = rng.uniform(lo, hi, size=(n, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    planes = np.zeros((2, n, 4), np.float32)
    planes[0, :, :3] = o
    planes[1, :, :3] = d
    planes[1, :, 3] = np.inf
    return planes


def _both(scene, rays=None, spp=0, max_depth=6):
    out = []
    for b in ("device", "host"):
        with PtSession(scene, abi.make_params(max_depth=max_depth, bvh_build=b)) as s:
            st = s.stats()
            r = {"blas": st["blas_nodes"], "tlas": st["tlas_nodes"], "tris": st["triangles"]}
            if rays is not None:
                r["closest"] = s.intersect(rays, any_hit=False)
                r["any"] = s.intersect(rays, any_hit=True)
            if spp:
                s.render_samples(5, spp)
                r["accum"] = s.sum_and_weight()
            out.append(r)
    return out


def _check(dev, host, exact_prims=True, t_ulps=0):
    assert (dev["blas"], dev["tlas"], dev["tris"]) == (host["blas"], host["tlas"], host["tris"])
    if "closest" in dev:
        (pd, idd, td), (ph, ih, th) = dev["closest"], host["closest"]
        d = np.abs(td.view(np.int32).astype(np.int64) - th.view(np.int32).astype(np.int64))
        assert d.max() <= t_ulps, (int(d.max()), int((d > 0).sum()))
        np.testing.assert_array_equal(pd == MISS, ph == MISS)
        if exact_prims:
            np.testing.assert_array_equal(pd, ph)
            np.testing.assert_array_equal(idd, ih)
        np.testing.assert_array_equal(dev["any"][0], host["any"][0])
    if "accum" in dev:
        np.testing.assert_array_equal(dev["accum"], host["accum"])


def test_cloud_matches_host_build():
    s = scenes.triangle_cloud(96, 64, 300_000)
    dev, host = _both(s, rays=_rays(262_144, 1, -0.5, 0.5), spp=4)
    assert dev["blas"] > 300_000 // 16
    _check(dev, host)


def test_instanced_scene_matches_host_build():
    s = scenes.instanced_materials(96, 64, n_instances=300, n_lights=16, subdivisions=3)
    dev, host = _both(s, rays=_rays(131_072, 2, -10.0, 10.0, radius=30.0), spp=2)
    assert dev["tlas"] > 0
    _check(dev, host)


def test_dense_instanced_scene_matches_host_build():
    """2,500 rotated, scaled copies of an icosphere crowded into a small box:
    a dense scene (the instances' boxes add up to well over 32 world boxes),
    so every instance becomes its BLAS's second-level frontier; the device
    makes those items (world boxes from the centre and |M| extents) exactly
    as the host does."""
    rng = np.random.default_rng(9)
    s = Scene(64, 48, fov=40.0)
    s.look_at((0.0, 0.0, 4.0), (0.0, 0.0, 0.0))
    mesh = s.add_mesh(*scenes.icosphere(3))
    mat = s.add_material(matte((0.6, 0.6, 0.6)))
    rot = scenes.random_rotations(rng, 2500)
    for k in range(2500):
        lin = rot[k] * rng.uniform(0.3, 0.5) * np.diag(rng.uniform(0.6, 1.4, 3))
        s.add_instance(mesh, mat, scenes.affine(lin, rng.uniform(-0.8, 0.8, 3)))
    s.add_point_light((0.0, 3.0, 3.0), 20.0)
    dev, host = _both(s, _rays(32768, 5), spp=2)
    _check(dev, host)
    assert dev["tlas"] > 0


@pytest.mark.parametrize("n", [1, 4, 5, 16, 17, 256, 257, 2048, 2049, 5000])
def test_mesh_sizes_around_builder_thresholds(n):
    # Leaf limits (4, 16), the subtree threshold (256) and the chunk size (2048).
    rng = np.random.default_rng(n)
    c = rng.uniform(-0.5, 0.5, size=(n, 1, 3))
    pos = (c + rng.normal(0, 0.02, size=(n, 3, 3))).reshape(-1, 3).astype(np.float32)
    idx = np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)
    s = Scene(32, 32)
    s.look_at((0, 0, 2.5), (0, 0, 0))
    m = s.add_material(matte((0.6, 0.6, 0.6)))
    s.add_mesh(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))  # empty mesh first
    s.add_instance(s.add_mesh(pos, idx), m)
    s.add_distant_light((0.3, -1, -0.2), 2.0)
    dev, host = _both(s, rays=_rays(65_536, 3 + n, -0.5, 0.5), spp=2)
    _check(dev, host)


def test_degenerate_and_offset_meshes():
    s = Scene(32, 32)
    s.look_at((1e4, 0, 1e4 + 4), (1e4, 0, 1e4))
    m = s.add_material(matte((0.5, 0.5, 0.5)))
    # 3000 copies of one triangle: every centroid coincides (median splits only).
    one = np.array([[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0]], np.float32) + np.float32(1e4)
    s.add_instance(s.add_mesh(np.tile(one, (3000, 1)), np.arange(9000, dtype=np.uint32).reshape(-1, 3)), m)
    # A flat sheet far from the origin (large exponents in the quantisation grid).
    rng = np.random.default_rng(9)
    c = np.concatenate([rng.uniform(-1, 1, size=(4000, 1, 2)), np.zeros((4000, 1, 1))], axis=2) + 1e4
    tri = (c + np.concatenate([rng.normal(0, 0.01, size=(4000, 3, 2)), np.zeros((4000, 3, 1))], axis=2))
    s.add_instance(s.add_mesh(tri.reshape(-1, 3).astype(np.float32), np.arange(12000, dtype=np.uint32).reshape(-1, 3)), m)
    # Triangles straddling zero on every axis (signed zeros in the boxes).
    z = np.array([[-0.0, 0.0, -0.0], [0.25, -0.0, 0.0], [0.0, 0.25, -0.0]], np.float32)
    s.add_instance(s.add_mesh(np.tile(z, (40, 1)) * np.repeat(np.arange(1, 41, dtype=np.float32), 3)[:, None],
                              np.arange(120, dtype=np.uint32).reshape(-1, 3)), m)
    s.add_point_light((1e4, 3, 1e4 + 3), 50.0)
    rays = _rays(65_536, 11, 1e4 - 1.0, 1e4 + 1.0, radius=4.0)
    rays[0, :, :3] += np.float32(1e4)
    d = np.float64(rng.uniform(1e4 - 1, 1e4 + 1, size=(65_536, 3))) - rays[0, :, :3]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays[1, :, :3] = d
    dev, host = _both(s, rays=rays, spp=2)
    # Coincident centroids end in median splits, which group primitives by
    # their order within the node (the host's swap partition and the
    # device's stable partition leave different orders): the trees have the
    # same shape but may group duplicates and coplanar triangles
    # differently, so the hit copy and, on 0.003% of rays here, the last
    # bit of t may differ.
    _check(dev, host, exact_prims=False, t_ulps=1)
    assert (dev["closest"][0] != MISS).mean() > 0.05


@pytest.mark.parametrize("bad", ["index", "vertex"])
def test_invalid_meshes_fail_like_the_host_build(bad):
    s = Scene(8, 8)
    m = s.add_material(matte((0.5, 0.5, 0.5)))
    good = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    s.add_instance(s.add_mesh(good, np.array([[0, 1, 2]], np.uint32)), m)
    pos = good.copy()
    idx = np.array([[0, 1, 2], [0, 2, 1]], np.uint32)
    if bad == "index":
        idx[1, 2] = 3
    else:
        pos[2, 1] = np.nan
    s.meshes.append((pos, idx, None))  # bypasses the Python-side index check
    s.add_instance(len(s.meshes) - 1, m)
    msgs = []
    for b in ("device", "host"):
        with pytest.raises(Exception) as e:
            PtSession(s, abi.make_params(bvh_build=b))
        msgs.append(str(e.value))
    want = "mesh 1 index out of range" if bad == "index" else "mesh 1 has a non-finite vertex"
    assert all(want in m for m in msgs), msgs
