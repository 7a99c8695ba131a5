"""Curves and Marschner hair on the GPU against the f64 oracle
(src/geometry/curves.rs rounded-cone segments through the same BVH / TLAS
as meshes, src/raytracer/pt/hair.rs and its branch of trace_full,
pt/mod.rs:737-781).

Ray batches: closest hits of random rays into a groomed sphere (20,000
cubic b-spline strands, 480,000 segments) agree with the oracle's ray for
ray, segment ids and distances. Images at the path tracer's tolerance
(tests/mc_parity.py): the furball, and a comb of tapered strands under a
rect light; the RIB route (Curves, Points, PxrMarschnerHair) renders the
same way."""
import numpy as np
import pytest

import oracle
from mc_parity import compare, render_quad
from rtcuda import PtSession, abi, scenes

pytestmark = pytest.mark.gpu


HAIR = ((0.4, 0.9, 1.8), 0.35, 0.32, 1.55)


def test_hair_bsdf_eval_matches_oracle():
    """Device hair f and pdf (f32) against the oracle's f64 on random
    fiber-frame queries."""
    from rtcuda import backend
    rng = np.random.default_rng(3)
    n = 20_000
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    h = rng.uniform(-1, 1, n)
    fg, pg = backend.hair_eval(HAIR, wo, wi, h)
    fo, po = np.zeros((n, 3)), np.zeros(n)
    for k in range(0, n, 2000):
        fo[k:k + 2000], po[k:k + 2000] = oracle.hair_eval(HAIR, wo[k:k + 2000], wi[k:k + 2000], h[k:k + 2000])
    scale_f, scale_p = np.maximum(np.abs(fo), 1e-3), np.maximum(po, 1e-3)
    assert np.quantile(np.abs(fg - fo) / scale_f, 0.999) < 1e-3
    assert np.quantile(np.abs(pg - po) / scale_p, 0.999) < 1e-3


def test_hair_sampling_matches_oracle():
    """Device hair::sample from the same PCG32 stream as the oracle's:
    the same directions (up to f32), and E[f / pdf] equal."""
    from rtcuda import backend
    for sin_to, h in ((0.3, -0.4), (-0.6, 0.8), (0.05, 0.0)):
        wo = np.array([sin_to, np.sqrt(1 - sin_to ** 2), 0.0])
        wg, fg, pg = backend.hair_sample(HAIR, wo, h, 11, 5, 40_000)
        wo_, fo, po = oracle.hair_sample(HAIR, wo, h, 11, 5, 40_000)
        same = np.linalg.norm(wg - wo_, axis=1) < 1e-3
        assert same.mean() > 0.99, same.mean()
        lum = lambda f: 0.2126 * f[:, 0] + 0.7152 * f[:, 1] + 0.0722 * f[:, 2]
        eg = np.where(pg > 0, lum(fg) / np.maximum(pg, 1e-30), 0).mean()
        eo = np.where(po > 0, lum(fo) / np.maximum(po, 1e-30), 0).mean()
        assert abs(eg - eo) < 0.01 * eo, (eg, eo)


@pytest.fixture(scope="module")
def fur():
    s = scenes.furball(64, 32, 20_000)
    return s, oracle.OracleScene(s)


def _rays_at_ball(n, seed):
    rng = np.random.default_rng(seed)
    centre = np.array([0.0, 1.32, 9.5])
    o = centre + rng.normal(size=(n, 3)) * 0.3 + np.array([0.0, 0.0, -6.0])
    tgt = centre + rng.normal(size=(n, 3)) * 0.7
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    planes = np.zeros((2, n, 4), np.float32)
    planes[0, :, :3] = o
    planes[1, :, :3] = d
    planes[1, :, 3] = np.inf
    return planes


def test_curve_ray_batch_matches_oracle(fur):
    s, o_s = fur
    planes = _rays_at_ball(65_536, 3)
    with PtSession(s, abi.make_params()) as g:
        gp, gi, gt = g.intersect(planes)
    op, oi, ot, _ = o_s.intersect(planes)
    hit = oi != 0xFFFFFFFF
    assert hit.mean() > 0.5
    curve_hits = hit & (oi == 0)
    assert curve_hits.mean() > 0.2            # the batch really meets the strands
    same = (gi == oi) & (gp == op)
    # f32 rounded cones against f64 ones: a ray that grazes a strand or
    # passes where two strands meet within f32 precision may pick the other.
    assert same.mean() > 0.995, same.mean()
    both = same & hit
    err = np.abs(gt[both] - ot[both]) / ot[both]
    assert np.quantile(err, 0.999) < 1e-4, np.quantile(err, 0.999)


def test_curve_any_hit_matches_oracle(fur):
    s, o_s = fur
    planes = _rays_at_ball(16_384, 4)
    with PtSession(s, abi.make_params()) as g:
        gh = g.intersect(planes, any_hit=True)[0]
    oh = o_s.intersect(planes, any_hit=True)[0]
    assert (gh == oh).mean() > 0.998


def test_furball_image_parity(fur):
    s, o_s = fur
    g, o, r, pr, st = render_quad(s, abi.make_params(max_depth=8), 32, 1024, oracle_scene=o_s)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res


def test_hair_comb_image_parity():
    s = scenes.Scene(48, 48, fov=30.0)
    s.look_at((0.0, 0.0, 4.0), (0.0, 0.0, 0.0))
    p0, p1, v0, v1 = [], [], [], []
    for k in range(60):
        x = -0.9 + 1.8 * k / 59
        for j in range(8):
            y0, y1 = -1 + 2 * j / 8, -1 + 2 * (j + 1) / 8
            r0, r1 = 0.03 * (1 - j / 8) + 0.006, 0.03 * (1 - (j + 1) / 8) + 0.006
            p0.append((x + 0.05 * np.sin(3 * y0), y0, 0.1 * np.cos(2 * x), r0))
            p1.append((x + 0.05 * np.sin(3 * y1), y1, 0.1 * np.cos(2 * x), r1))
            v0.append(j / 8)
            v1.append((j + 1) / 8)
    hm = s.add_material(scenes.marschner_hair(color=(0.7, 0.5, 0.3), roughness=0.25, azimuthal_roughness=0.4))
    s.add_instance(s.add_curves(p0, p1, v0, v1), hm)
    back = s.add_material(scenes.matte((0.5, 0.5, 0.5)))
    s.add_instance(s.add_mesh(*scenes.quad((-3, -3, -1), (6, 0, 0), (0, 6, 0))), back)
    s.add_rect_light((-1, 2, 1), (2, 0, 0), (0, 0, 1), 10.0)
    g, o, r, pr, _ = render_quad(s, abi.make_params(max_depth=8), 32, 1024)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res


def test_rib_curves_points_hair_parity():
    from rtcuda.rib import load_rib_string
    s = load_rib_string("""
Format 48 32 1
Projection "perspective" "fov" [40]
WorldBegin
  Light "PxrDomeLight" "sky" "intensity" [0.5]
  Bxdf "PxrMarschnerHair" "h" "roughness" [0.3] "color" [0.6 0.4 0.2]
  Basis "catmull-rom" 1 "catmull-rom" 1
  Curves "cubic" [5 5 5] "nonperiodic" "P" [-1 -1 4  -0.5 -0.5 4.2  0 0 4  0.5 0.5 4.2  1 1 4
                                          -1 1 4  -0.5 0.5 4.1  0 0 4.3  0.5 -0.5 4.1  1 -1 4
                                          -1 0 4.5  -0.5 0.2 4.5  0 0 4.5  0.5 -0.2 4.5  1 0 4.5] "width" [0.08 0.02]
  Bxdf "PxrSurface" "p" "diffuseColor" [0.8 0.3 0.2]
  Points "P" [-0.6 -0.6 3.5  0.6 0.6 3.5  0.6 -0.6 3.5] "width" [0.2 0.3 0.25]
WorldEnd
""")
    g, o, r, pr, _ = render_quad(s, abi.make_params(max_depth=8), 32, 1024)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res


def test_furball_same_seed_bitwise(fur):
    s, _ = fur
    imgs = []
    for _ in range(2):
        with PtSession(s, abi.make_params(max_depth=8)) as g:
            g.render_samples(0, 4)
            imgs.append(g.image())
    assert np.array_equal(imgs[0], imgs[1])
