"""The path tracer against the f64 oracle at its stated tolerance, on every
configured workload, plus the device functions under the image one at a
time.

Images (tests/mc_parity.py): the GPU render's relMSE against a high-spp
oracle render lies within the Monte Carlo confidence interval of the
relMSE of an independent oracle render at the same spp, and the GPU image
has the mean of the oracle's render of the same samples. The configurations run at reduced
resolution with their own meshes, materials, lights and depths; the oracle
renders a strided subset of the pixels where a full frame is too slow:
  C1 Cornell box 256x256 x 16 spp, depth 8 (the full frame);
  C2 1M-triangle cloud under a distant light, 192x108 x 16 spp, depth 8;
  C3 1,000 instances of icospheres subdivided 5 times and 128x128 fBm grids,
     GGX / Oren-Nayar / rough glass, 64 point lights, 128x72 x 64 spp, depth 12;
  C4 two rooms, light in the unseen one, 128x72 x 64 spp, depth 16;
  C5 the 772,001-instance forest with leaf cutouts and 1,200 point lights,
     64x36 x 32 spp, depth 10;
  and a Cornell box whose small, bright light makes paths trip the firefly
  clamp (src/raytracer/pt/mod.rs:28-29, 90-93).
Functions: the device PCG32 stream bit for bit (sampler.rs:24-42), the
light BVH's pick and pmf (light_sampler.rs:150-238) on the C3 and C5 light
sets, and the shadow transmittance through the forest's cutouts
(pt/mod.rs:1254-1306).
"""
import numpy as np
import pytest

import oracle
from mc_parity import compare, render_quad
from rtcuda import PtSession, abi, backend, scenes

pytestmark = pytest.mark.gpu


def _image_parity(s, depth, spp, ref_spp, stride, oracle_scene=None, **kw):
    p = abi.make_params(max_depth=depth, **kw)
    g, o, r, pr, st = render_quad(s, p, spp, ref_spp, pixel_stride=stride, oracle_scene=oracle_scene)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res
    return res, st


def test_c1_cornell_full_frame():
    _image_parity(scenes.cornell_box(), 8, 16, 512, 1)


def test_c2_triangle_cloud():
    _image_parity(scenes.triangle_cloud(192, 108), 8, 16, 256, 2)


def test_c3_instanced_materials_full_meshes():
    s = scenes.instanced_materials(128, 72)
    _, st = _image_parity(s, 12, 64, 1024, 4)
    assert st["shadow_rays"] > 0


def test_c4_two_rooms():
    _image_parity(scenes.two_rooms(128, 72), 16, 64, 2048, 4)


@pytest.fixture(scope="module")
def forest():
    s = scenes.forest(64, 36)
    return s, oracle.OracleScene(s)


def test_c5_forest(forest):
    s, o_s = forest
    assert any(m["presence"] < 1.0 for m in s.materials)
    _image_parity(s, 10, 32, 256, 4, oracle_scene=o_s)


def test_c5_forest_same_seed_bitwise(forest):
    s, _ = forest
    imgs = []
    for _ in range(2):
        with PtSession(s, abi.make_params(max_depth=10)) as g:
            g.render_samples(5, 3)
            imgs.append(g.image())
    assert np.array_equal(imgs[0], imgs[1])


def test_firefly_clamp_parity():
    """A 0.1 x 0.1 light of radiance (425, 300, 100) (luminance 312) in the
    Cornell box: samples that see it, and NEE from surfaces near it, exceed
    the luminance clamp of 60 and are scaled down to it."""
    s = scenes.cornell_box(64, 64, light_size=0.1, light_radiance=(425.0, 300.0, 100.0))
    means = {}
    for clamp in (60.0, 1e30):
        with PtSession(s, abi.make_params(max_depth=8, firefly_clamp=clamp)) as g:
            g.render_samples(0, 64)
            means[clamp] = g.image().mean()
    assert means[60.0] < 0.97 * means[1e30], means   # the clamp really acts
    _image_parity(s, 8, 64, 1024, 1)


def test_pcg_stream_bit_exact():
    rng = np.random.default_rng(5)
    pixels = rng.integers(0, 3840 * 2160, 2048, dtype=np.uint64)
    samples = rng.integers(0, 1 << 24, 2048, dtype=np.uint64)
    pixels[:4] = [0, 1, 3840 * 2160 - 1, 12345]
    samples[:4] = [0, 0, 31, 1 << 23]
    dev = backend.pcg_streams(pixels, samples, 48)
    for k in range(len(pixels)):
        ref = oracle.pcg_stream(int(pixels[k]), int(samples[k]), 48)
        assert np.array_equal(dev[k], ref), k


def _light_parity(s, lo, hi, n_points=48, per_point=512):
    rng = np.random.default_rng(9)
    o_s = oracle.OracleScene(s)
    n_lights = len(s.lights)
    pts = rng.uniform(lo, hi, size=(n_points, 3)).astype(np.float32)
    with PtSession(s, abi.make_params(max_depth=4)) as g:
        # pmf of every light at every point, and its normalisation
        P = np.repeat(pts, n_lights, 0)
        L = np.tile(np.arange(n_lights, dtype=np.uint32), n_points)
        dpmf = g.light_pmf(P, L).astype(np.float64)
        opmf = np.array([o_s.light_pmf(P[i].astype(np.float64), int(L[i])) for i in range(len(P))])
        np.testing.assert_allclose(dpmf, opmf, rtol=2e-4, atol=1e-9)
        np.testing.assert_allclose(dpmf.reshape(n_points, n_lights).sum(1), 1.0, rtol=2e-4)
        # picks at stratified uniforms
        u = ((np.arange(per_point) + 0.5) / per_point).astype(np.float32)
        P2 = np.repeat(pts, per_point, 0)
        U2 = np.tile(u, n_points)
        dl, dp = g.light_sample(P2, U2)
        consistent = g.light_pmf(P2, dl)
    ol = np.empty(len(P2), np.uint32)
    op = np.empty(len(P2))
    for i in range(len(P2)):
        ol[i], op[i] = o_s.light_sample(P2[i].astype(np.float64), float(U2[i]))
    agree = dl == ol
    # Disagreement only where f32 and f64 split a node's interval differently,
    # i.e. at a few uniforms per point next to a split point.
    assert agree.mean() > 0.995, agree.mean()
    np.testing.assert_allclose(dp[agree], op[agree], rtol=2e-4)
    np.testing.assert_allclose(dp, consistent, rtol=2e-4)   # sample's pmf == pmf()
    return n_lights


def test_light_bvh_instanced_materials_lights():
    s = scenes.instanced_materials(8, 8, subdivisions=1, grid=4)
    assert _light_parity(s, (-12, 0, -12), (12, 8, 12)) == 64


def test_light_bvh_forest_lights(forest):
    s, _ = forest
    assert _light_parity(s, (-500, -20, -500), (500, 40, 500), n_points=24, per_point=256) == 1200


def test_shadow_transmittance_through_cutouts(forest):
    """Shadow rays from points among the trees toward the scene's lights:
    the device's one-traversal transmittance against the reference's
    closest-hit segment loop."""
    s, o_s = forest
    rng = np.random.default_rng(17)
    n = 8192
    lights = np.array([l["p"] for l in s.lights], np.float64)
    org = np.stack([rng.uniform(-150, 150, n), rng.uniform(0, 14, n), rng.uniform(-150, 150, n)], 1)
    tgt = lights[rng.integers(0, len(lights), n)]
    # keep each ray within ~60 m of its origin, toward a light
    dvec = tgt - org
    dist = np.linalg.norm(dvec, axis=1)
    d = dvec / dist[:, None]
    tmax = np.minimum(dist, 60.0)
    planes = np.zeros((2, n, 4), np.float32)
    planes[0, :, :3] = org
    planes[1, :, :3] = d
    planes[1, :, 3] = tmax
    with PtSession(s, abi.make_params(max_depth=4)) as g:
        dev = g.transmittance(planes).astype(np.float64)
    ref = o_s.transmittance(planes)[:, 0]
    assert 0.05 < (ref > 0).mean() < 0.95          # the set crosses the canopy
    close = np.abs(dev - ref) <= 1e-6 + 1e-5 * ref
    # A ray that grazes a leaf's edge may count it on one side only.
    assert close.mean() > 0.99, close.mean()
    assert abs(dev.mean() - ref.mean()) <= 0.01 * ref.mean() + 1e-6
