"""GPU traversal parity against the f64 oracle, through the C ABI.

Closest hit must agree with the oracle on primitive and instance id; a
disagreement is allowed only at a near-tie, i.e. where the two answers are
within |dt|/t < 1e-4 of each other, or where the ray passes within 1e-5
(relative, in barycentric units) of an edge of the triangle that decides
the outcome -- or, for a grazing triangle, within 2 f32 ulps of the ray
origin's coordinates of that edge, measured across the ray -- so the f32
watertight test and the f64 Möller–Trumbore test may legitimately
disagree. t must agree to 1e-5 relative on agreeing hits
(all but 1 in 10^4; grazing hits within 1e-4).
"""
import numpy as np
import pytest

import oracle
from rtcuda import PtSession, scene, scenes

pytestmark = pytest.mark.gpu

T_TIE = 1e-4
EDGE = 1e-5
EDGE_ULPS = 2.0


def _bary(tri, o, d):
    """The smallest barycentric coordinate of the ray's crossing of the
    triangle's plane (negative outside), in f64."""
    m = _edge_metrics(tri, o, d)
    return None if m is None else m[0]


def _edge_metrics(tri, o, d):
    v0, v1, v2 = tri
    e1, e2 = v1 - v0, v2 - v0
    p = np.cross(d, e2)
    det = e1 @ p
    if abs(det) < 1e-300:
        return None
    tv = o - v0
    u = (tv @ p) / det
    q = np.cross(tv, e1)
    v = (d @ q) / det
    m = min(u, v, 1 - u - v)
    # |m| |det| / (longest edge): the crossing's distance from the nearest
    # edge line, measured across the ray (times |d|), in world units.
    longest = max(np.linalg.norm(e1), np.linalg.norm(e2), np.linalg.norm(v2 - v1))
    return m, abs(m) * abs(det) / max(longest, 1e-300)


def _near_edge(tri, o, d):
    """Within EDGE of an edge in barycentric units, or (grazing triangles,
    whose small determinant magnifies f32 rounding in the barycentrics)
    within EDGE_ULPS f32 ulps of the ray origin's largest coordinate of an
    edge, measured across the ray."""
    m = _edge_metrics(tri, o, d)
    if m is None:
        return False
    ulp = np.spacing(np.float32(np.abs(o).max()))
    return abs(m[0]) < EDGE or m[1] < EDGE_ULPS * float(ulp)


def _check_closest(s, planes, gp, gi, gt, op, oi, ot, tri_of):
    n = planes.shape[1]
    o = planes[0, :, :3].astype(np.float64)
    d = planes[1, :, :3].astype(np.float64)
    bad = []
    agree = (gp == op) & (gi == oi)
    hit = agree & (op != 0xFFFFFFFF)
    # f32 t vs f64 t: relative 1e-5 (absolute for hits close to the origin)
    # for all but 1 in 10^4 hits; grazing hits (small determinant) amplify
    # the f32 rounding of T / det, so every hit only within 1e-4.
    err = np.abs(gt[hit].astype(np.float64) - ot[hit]) / np.maximum(ot[hit], 1.0)
    if err.size:
        assert np.quantile(err, 0.9999) < 1e-5 and err.max() < 1e-4, (np.quantile(err, 0.9999), err.max())
    for k in np.nonzero(~agree)[0]:
        tg = np.inf if gp[k] == 0xFFFFFFFF else float(gt[k])
        to = float(ot[k])
        if np.isfinite(tg) and np.isfinite(to) and abs(tg - to) / to < T_TIE:
            continue
        near_edge = False
        for p_, i_ in ((gp[k], gi[k]), (op[k], oi[k])):
            if p_ != 0xFFFFFFFF and _near_edge(tri_of(i_, p_), o[k], d[k]):
                near_edge = True
        if not near_edge:
            bad.append((int(k), int(gp[k]), int(op[k]), tg, to))
    assert not bad, f"{len(bad)} non-tie mismatches of {n}: {bad[:5]}"
    return int((~agree).sum())


def _tri_lookup(s):
    inst = s.instance_array()

    def tri_of(i, p):
        pos, idx, _ = s.meshes[inst["mesh"][i]]
        xf = inst["xf"][i].reshape(3, 4)
        v = pos[idx[p]].astype(np.float64)
        return v @ xf[:, :3].T + xf[:, 3]
    return tri_of


@pytest.fixture(scope="module")
def cloud():
    s = scene.Scene(16, 16)
    s.add_instance(s.add_mesh(*scenes.triangle_cloud_mesh(50_000, seed=11)), s.add_material(scene.matte((0.5,) * 3)))
    rays = scenes.triangle_cloud_rays(65_536, seed=12)
    return s, rays


def test_closest_hit_matches_oracle(cloud):
    s, rays = cloud
    op, oi, ot, _ = oracle.OracleScene(s).intersect(rays)
    with PtSession(s) as g:
        gp, gi, gt = g.intersect(rays)
    assert (op != 0xFFFFFFFF).mean() > 0.5   # the set really hits the cloud
    _check_closest(s, rays, gp, gi, gt, op, oi, ot, _tri_lookup(s))


def test_any_hit_matches_oracle(cloud):
    s, rays = cloud
    r = rays.copy()
    r[1, :, 3] = 2.0   # finite segment: origins sit on the radius-2 sphere
    o_s = oracle.OracleScene(s)
    ohit = o_s.intersect(r, any_hit=True)[0].astype(bool)
    op, oi, ot, _ = o_s.intersect(r)
    with PtSession(s) as g:
        ghit, _, _ = g.intersect(r, any_hit=True)
    diff = np.nonzero(ghit != ohit)[0]
    assert np.array_equal(ohit, op != 0xFFFFFFFF)
    # Disagreement only where the oracle's closest hit is at the segment end
    # or grazes an edge.
    tri_of = _tri_lookup(s)
    for k in diff:
        if op[k] != 0xFFFFFFFF and abs(ot[k] - 2.0) / 2.0 < T_TIE:
            continue
        if op[k] != 0xFFFFFFFF:
            m = _bary(tri_of(oi[k], op[k]), r[0, k, :3].astype(np.float64), r[1, k, :3].astype(np.float64))
            assert m is not None and abs(m) < EDGE, (k, m)
        else:
            pytest.fail(f"ray {k}: GPU any-hit with no oracle hit")


def test_instances_match_oracle():
    """Cornell scene: 7 instances (two scaled + rotated), rays from the camera region."""
    s = scenes.cornell_box(8, 8)
    rng = np.random.default_rng(5)
    n = 20_000
    o = rng.uniform(-0.9, 0.9, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    planes = np.zeros((2, n, 4), np.float32)
    planes[0, :, :3] = o
    planes[1, :, :3] = d
    planes[1, :, 3] = np.inf
    op, oi, ot, _ = oracle.OracleScene(s).intersect(planes)
    with PtSession(s) as g:
        gp, gi, gt = g.intersect(planes)
    _check_closest(s, planes, gp, gi, gt, op, oi, ot, _tri_lookup(s))


def test_empty_batch_and_miss_everything():
    s = scenes.cornell_box(8, 8)
    with PtSession(s) as g:
        planes = np.zeros((2, 0, 4), np.float32)
        assert g.intersect(planes)[0].size == 0
        planes = np.zeros((2, 64, 4), np.float32)
        planes[0, :, 2] = 10.0
        planes[1, :, 2] = 1.0          # pointing away from the box
        planes[1, :, 3] = np.inf
        p, i, t = g.intersect(planes)
        assert (p == 0xFFFFFFFF).all() and np.isinf(t).all()


def test_full_traversal_stress_set():
    """The traversal-stress configuration at its stated size: 4,194,304
    seeded rays (origins on the radius-2 sphere, aimed into the cube) into
    the 1,000,000-triangle cloud, closest hit and any hit, checked ray for
    ray against the f64 oracle with the near-tie / edge rule above; the
    mismatch count is reported."""
    s = scene.Scene(16, 16)
    s.add_instance(s.add_mesh(*scenes.triangle_cloud_mesh(1_000_000)), s.add_material(scene.matte((0.5,) * 3)))
    rays = scenes.triangle_cloud_rays(4_194_304)
    op, oi, ot, _ = oracle.OracleScene(s).intersect(rays)
    with PtSession(s) as g:
        gp, gi, gt = g.intersect(rays)
        ghit, _, _ = g.intersect(rays, any_hit=True)
    tri_of = _tri_lookup(s)
    mismatches = _check_closest(s, rays, gp, gi, gt, op, oi, ot, tri_of)
    print(f"closest hit: {mismatches} near-tie / edge mismatches of {rays.shape[1]}")
    assert mismatches < 1e-3 * rays.shape[1]
    ohit = op != 0xFFFFFFFF
    for k in np.nonzero(ghit.astype(bool) != ohit)[0]:
        o_k, d_k = rays[0, k, :3].astype(np.float64), rays[1, k, :3].astype(np.float64)
        assert any(p_ != 0xFFFFFFFF and _near_edge(tri_of(i_, p_), o_k, d_k)
                   for p_, i_ in ((gp[k], gi[k]), (op[k], oi[k]))), k
