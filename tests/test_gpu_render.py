"""GPU path tracer against the f64 oracle, through the C ABI.

The GPU draws its uniforms as (u32 >> 8) * 2^-24 in f32 while the oracle
uses u32 / 2^32 in f64 (as the reference's Metal and CPU paths do), so
image parity is statistical: per-channel means within 3% and RMSE bounded
by Monte Carlo noise, the reference's own CPU-vs-GPU criterion
(tests/metal_pt_tests.rs:42-64). Within the GPU path, results are bitwise
reproducible for a seed.
"""
import numpy as np
import pytest

import oracle
from rtcuda import PtSession, abi, backend, render_pt_film, scene, scenes

pytestmark = pytest.mark.gpu


def _stat_parity(cpu, gpu, mean_tol, rmse_tol):
    mc, mg = cpu.reshape(-1, 3).mean(0), gpu.reshape(-1, 3).mean(0)
    for c, g in zip(mc, mg):
        assert abs(c - g) / max(abs(c), 0.02) < mean_tol, (mc, mg)
    e = np.sqrt(((cpu - gpu) ** 2).mean())
    assert e < rmse_tol, e
    return mc, mg, e


@pytest.fixture(scope="module")
def cornell():
    s = scenes.cornell_box(64, 64)
    p = abi.make_params(max_depth=8)
    rgb, _, _ = oracle.OracleScene(s).render(p, 0, 64)
    return s, p, rgb.reshape(64, 64, 3) / 64


def test_cornell_statistical_parity(cornell):
    s, p, cpu = cornell
    with PtSession(s, p) as g:
        g.render_samples(0, 64)
        gpu = g.image()
        st = g.stats()
    _stat_parity(cpu, gpu, 0.03, 0.10)
    assert st["extension_rays"] > 64 * 64 * 64 and st["shadow_rays"] > 0


def test_bitwise_reproducible(cornell):
    s, p, _ = cornell
    out = []
    for _ in range(2):
        with PtSession(s, p) as g:
            g.render_samples(0, 8)
            out.append(g.sum_and_weight())
    assert np.array_equal(out[0], out[1])


def test_sample_ranges_add_up(cornell):
    s, p, _ = cornell
    with PtSession(s, p) as g:
        g.render_samples(0, 8)
        full = g.sum_and_weight()
        g.reset()
        g.render_samples(0, 3)
        g.render_samples(3, 5)
        parts = g.sum_and_weight()
    assert np.allclose(full, parts, rtol=1e-12, atol=1e-12)
    assert (full[..., 3] == 8).all()


def test_slab_size_does_not_change_result(cornell):
    s, _, _ = cornell
    res = []
    for cap in (0, 64 * 64):   # 8 samples per slab vs one sample per slab
        with PtSession(s, abi.make_params(max_depth=8, max_paths=cap)) as g:
            g.render_samples(0, 8)
            res.append(g.sum_and_weight())
    assert np.allclose(res[0], res[1], rtol=1e-12, atol=1e-12)


def test_checkpoint_resume(cornell, tmp_path):
    s, p, _ = cornell
    ck = str(tmp_path / "ck.bin")
    with PtSession(s, p) as g:
        g.render_samples(0, 4)
        g.checkpoint_save(ck)
    with PtSession(s, p) as g:
        assert g.checkpoint_load(ck) == 4
        g.render_samples(4, 4)
        resumed = g.sum_and_weight()
    with PtSession(s, p) as g:
        g.render_samples(0, 8)
        straight = g.sum_and_weight()
    assert np.allclose(resumed, straight, rtol=1e-12, atol=1e-12)
    with PtSession(scenes.cornell_box(32, 32), p) as g:
        with pytest.raises(backend.RtError):
            g.checkpoint_load(ck)
    with open(ck, "r+b") as f:
        f.truncate(100)
    with PtSession(s, p) as g:
        with pytest.raises(backend.RtError):
            g.checkpoint_load(ck)


def test_aov_film(cornell):
    s, _, _ = cornell
    film = render_pt_film(s, 8, max_depth=8)
    # Back wall above the boxes (row 20, column 40): white albedo, normal +z,
    # depth = distance from the eye to about (0.47, 0.64, -1), i.e. ~4.96.
    c = film["albedo"][20, 40]
    assert np.allclose(c, 0.73, atol=1e-5)
    n = film["normal"][20, 40]
    assert n[2] > 0.999
    assert 4.9 < film["depth"][20, 40, 0] < 5.05
    assert film["id"][20, 40, 0] == 1 and film["id"][20, 40, 1] == 1.0
    # Left wall: red albedo; diffuse AOV equals beauty for all-diffuse scenes.
    assert np.allclose(film["albedo"][32, 8], (0.63, 0.065, 0.05), atol=1e-5)
    assert np.allclose(film["diffuse"], film["beauty"], rtol=1e-4, atol=1e-5)


def test_triangle_cloud_render_parity():
    s = scenes.triangle_cloud(64, 36, n_tris=50_000)
    p = abi.make_params(max_depth=8)
    spp = 64
    cpu = oracle.OracleScene(s).render(p, 0, spp)[0].reshape(36, 64, 3) / spp
    with PtSession(s, p) as g:
        g.render_samples(0, spp)
        gpu = g.image()
    _stat_parity(cpu, gpu, 0.03, 0.05)


FURNACE_N = 10_000_000


@pytest.mark.parametrize("name,mat,eta", [
    ("lambert", scene.matte((1.0, 1.0, 1.0)), 1.5),
    ("oren_nayar", scene.matte((1.0, 1.0, 1.0), sigma=0.5), 1.5),
    ("ggx_conductor", scene.ggx_conductor(1.0, 0.3), 1.5),
    ("ggx_plastic", scene.ggx_floor((1.0, 1.0, 1.0), 0.3), 1.5),
    ("rough_dielectric", scene.rough_dielectric(1.5, 0.05), 1.5),
])
def test_white_furnace_per_lobe(name, mat, eta):
    """GPU f32 BSDF energy vs the f64 oracle within 1e-3 per lobe (1e7 samples each)."""
    wo = np.array([0.2, 0.1, 0.97])
    wo /= np.linalg.norm(wo)
    g, _ = backend.bsdf_furnace(mat, wo, eta, FURNACE_N, seed=1)
    m = abi.RtMaterialDesc()
    for k, v in mat.items():
        setattr(m, k, abi.c_double3(*v) if isinstance(v, tuple) else v)
    c, _ = oracle.bsdf_furnace(m, wo, eta, FURNACE_N)
    assert abs(g - c) < 1e-3, (name, g, c)
    if name == "lambert":
        assert abs(g - 1.0) < 1e-3


def test_constant_dome_furnace_and_oracle():
    # Lambertian sphere of albedo 0.5 in a unit constant dome: surface pixels
    # converge to 0.5, missed pixels show the dome; GPU and oracle agree.
    from rtcuda.scene import Scene, matte
    s = Scene(32, 32, fov=30.0)
    s.look_at((0, 0, -4.0), (0, 0, 0))
    pos, idx, nrm = scenes.icosphere(4)
    s.add_instance(s.add_mesh(pos, idx, normals=nrm), s.add_material(matte((0.5, 0.5, 0.5))))
    s.add_dome_light(1.0, (1.0, 1.0, 1.0))
    p = abi.make_params(max_depth=8)
    spp = 1024
    with PtSession(s, p) as g:
        g.render_samples(0, spp)
        img = g.image()
    np.testing.assert_allclose(img[0, 0], 1.0, rtol=1e-6)
    np.testing.assert_allclose(img[12:20, 12:20].mean((0, 1)), 0.5, rtol=0.01)
    cpu = oracle.OracleScene(s).render(p, 0, 256)[0].reshape(32, 32, 3) / 256
    np.testing.assert_allclose(img.mean((0, 1)), cpu.mean((0, 1)), rtol=0.01)


def test_environment_map_dome_matches_oracle():
    # A dome with a lat-long map (a bright patch on a dim sky): camera misses
    # show the map, and the lit sphere agrees with the oracle (envmap.rs
    # importance sampling for NEE, MIS-weighted misses).
    from rtcuda.scene import Scene, matte
    env = np.full((16, 32, 3), 0.2, np.float32)
    env[3:6, 10:16] = (20.0, 16.0, 10.0)
    s = Scene(32, 32, fov=50.0)
    s.look_at((0, 0, -3.0), (0, 0, 0))
    pos, idx, nrm = scenes.icosphere(4)
    s.add_instance(s.add_mesh(pos, idx, normals=nrm), s.add_material(matte((0.6, 0.6, 0.6))))
    s.add_dome_light(1.5, (1.0, 1.0, 1.0), env=env)
    p = abi.make_params(max_depth=8)
    with PtSession(s, p) as g:
        g.render_samples(0, 1024)
        img = g.image()
    cpu = oracle.OracleScene(s).render(p, 0, 1024)[0].reshape(32, 32, 3) / 1024
    np.testing.assert_allclose(img[0, 0], cpu[0, 0], rtol=1e-3)   # a miss: map * intensity
    np.testing.assert_allclose(img.mean((0, 1)), cpu.mean((0, 1)), rtol=0.02)
    np.testing.assert_allclose(img[10:22, 10:22].mean((0, 1)), cpu[10:22, 10:22].mean((0, 1)), rtol=0.03)
