"""Analytic quadrics in the f64 oracle, pinned by the reference's own unit
tests of its legacy primitives (src/geometry/sphere.rs:131-168,
cylinder.rs:125-153, cone.rs:146-168, extra.rs:737-786), and the scene-level
rule that quadrics are scanned before the meshes (src/scene/mod.rs:105-146)."""
import numpy as np

import oracle
from rtcuda import abi, scene


def _q(kind, params, xf=None):
    d = abi.RtQuadricDesc()
    d.object_to_world = (abi.C.c_double * 12)(*(scene.affine() if xf is None else xf))
    pr = list(params) + [0.0] * (8 - len(params))
    d.params = (abi.C.c_double * 8)(*pr)
    d.type = kind
    d.material_id = 0
    return d


def _hit(desc, o, d):
    return oracle.quadric_intersect(desc, np.array([o], float), np.array([d], float))[0]


def test_sphere_hit_miss_and_st():
    s = _q(abi.QUADRIC_SPHERE, [1.0, -1.0, 1.0, 360.0])
    h = _hit(s, (0, 0, -5), (0, 0, 1))
    assert h[0] > 0.0
    h = _hit(s, (-5, 0, 0), (1, 0, 0))            # equator at (-1, 0, 0)
    assert abs(h[7] - 0.5) < 1e-9 and abs(h[8] - 0.5) < 1e-9
    assert abs(h[9] - 1.0 / np.sqrt(2.0 * np.pi * 2.0)) < 1e-9
    assert _hit(s, (5, 5, -5), (0, 0, 1))[0] < 0.0


def test_cylinder_and_cone():
    c = _q(abi.QUADRIC_CYLINDER, [1.0, -1.0, 1.0, 360.0])
    assert _hit(c, (2, 0, 0), (-1, 0, 0))[0] > 0.0
    assert _hit(c, (5, 5, -5), (0, 0, 1))[0] < 0.0
    k = _q(abi.QUADRIC_CONE, [2.0, 1.0, 360.0])
    assert _hit(k, (0, 0, -5), (0, 0, 1))[0] > 0.0
    assert _hit(k, (5, 5, -5), (0, 0, 1))[0] < 0.0


def test_quartic_known_roots_and_torus_axis_ray():
    np.testing.assert_allclose(oracle.solve_quartic([1.0, -10.0, 35.0, -50.0, 24.0]), [1, 2, 3, 4], atol=1e-6)
    t = _q(abi.QUADRIC_TORUS, [2.0, 0.5, 0.0, 360.0, 360.0])
    h = _hit(t, (-5, 0, 0), (1, 0, 0))
    assert abs(h[0] - 2.5) < 1e-6


def test_disk_paraboloid_hyperboloid():
    d = _q(abi.QUADRIC_DISK, [1.0, 2.0, 360.0])
    assert abs(_hit(d, (0.5, 0.5, -3), (0, 0, 1))[0] - 4.0) < 1e-9
    part = _q(abi.QUADRIC_DISK, [1.0, 2.0, 90.0])
    assert _hit(part, (0.5, -0.5, -3), (0, 0, 1))[0] < 0.0   # phi = 315 > 90
    par = _q(abi.QUADRIC_PARABOLOID, [1.0, 0.0, 1.0, 360.0])
    assert abs(_hit(par, (0.5, 0, -2), (0, 0, 1))[3] - 0.25) < 1e-9
    hyp = _q(abi.QUADRIC_HYPERBOLOID, [1.0, 0.0, -1.0, 1.0, 0.0, 1.0, 360.0])
    assert abs(_hit(hyp, (-5, 0, 0), (1, 0, 0))[0] - 4.0) < 1e-9


def test_transformed_quadric_world_distance():
    """t is the world distance: a unit sphere scaled by 2 and moved to z = 10
    is met at t = 8 by a ray from the origin along +z."""
    s = _q(abi.QUADRIC_SPHERE, [1.0, -1.0, 1.0, 360.0], scene.affine(np.eye(3) * 2.0, (0, 0, 10)))
    h = _hit(s, (0, 0, 0), (0, 0, 1))
    assert abs(h[0] - 8.0) < 1e-9
    np.testing.assert_allclose(h[4:7], [0, 0, -1], atol=1e-12)


def test_scene_scans_quadrics_before_meshes():
    """A quadric in front of a mesh wins; behind it, the mesh wins."""
    s = scene.Scene(4, 4)
    m = s.add_material(scene.matte((0.5,) * 3))
    quad = s.add_mesh([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], [[0, 1, 2], [0, 2, 3]])
    s.add_instance(quad, m, scene.affine(np.eye(3), (0, 0, 5)))
    s.add_quadric(abi.QUADRIC_SPHERE, [0.5, -0.5, 0.5, 360.0], m, scene.affine(np.eye(3), (0, 0, 3)))
    s.add_quadric(abi.QUADRIC_DISK, [0.0, 1.0, 360.0], m, scene.affine(np.eye(3), (0, 0, 8)))
    o_s = oracle.OracleScene(s)
    planes = np.zeros((2, 2, 4), np.float32)
    planes[0, 0, :3] = (0, 0, 0)
    planes[0, 1, :3] = (0.9, 0.9, 0)          # misses the sphere, hits the mesh
    planes[1, :, :3] = (0, 0, 1)
    planes[1, :, 3] = np.inf
    prim, inst, t, _ = o_s.intersect(planes)
    assert inst[0] == 0x80000000 and abs(t[0] - 2.5) < 1e-9
    assert inst[1] == 0 and abs(t[1] - 5.0) < 1e-9
    # The disk behind the mesh never wins; any-hit sees both kinds.
    hit = o_s.intersect(planes, any_hit=True)[0]
    assert hit.all()
