"""Pins the f64 oracle against the reference's own known-answer tests.

Each test restates a unit or scene test of anders94/render.rs with the same
inputs and thresholds (file:line in each docstring), plus the published
PCG32 reference vector. CPU only.
"""
import numpy as np
import pytest

import oracle
from rtcuda import abi, scene, scenes

# pcg32 demo output for pcg32_srandom_r(42, 54) (O'Neill, pcg-c-basic):
# the reference's Pcg32::new(seed, stream) is that generator.
PCG32_42_54 = [0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293, 0xbfa4784b, 0xcbed606e]


def test_pcg32_published_vector():
    assert oracle.pcg_new_stream(42, 54, 6).tolist() == PCG32_42_54


def test_pcg32_uniform_mean():
    """sampler.rs:64-71: mean of 100k uniforms from Pcg32::new(42, 54) within 0.005."""
    u = oracle.pcg_new_stream(42, 54, 100_000).astype(np.float64) / 2.0 ** 32
    assert abs(u.mean() - 0.5) < 0.005


def test_pcg32_per_pixel_sample_streams():
    """sampler.rs:73-88: same (pixel, sample) -> same stream; other sample -> different."""
    a = oracle.pcg_stream(7, 3, 8)
    b = oracle.pcg_stream(7, 3, 8)
    c = oracle.pcg_stream(7, 4, 8)
    assert (a == b).all() and not (a == c).all()


def _lcg_soup(n_tris=500, n_rays=2000):
    """The reference's seeded soup (bvh.rs:403-425): LCG 0x12345678, values in [-4, 4)."""
    state = 0x12345678
    M = (1 << 64) - 1

    def rnd():
        nonlocal state
        state = (state * 6364136223846793005 + 1442695040888963407) & M
        return ((state >> 11) / float(1 << 53)) * 8.0 - 4.0

    tris = []
    for _ in range(n_tris):
        base = np.array([rnd(), rnd(), rnd()])
        tris.append([base, base + np.array([rnd(), rnd(), rnd()]) * 0.2,
                     base + np.array([rnd(), rnd(), rnd()]) * 0.2])
    rays = []
    for _ in range(n_rays):
        o = np.array([rnd(), rnd(), rnd()])
        d = np.array([rnd(), rnd(), rnd()])
        if np.linalg.norm(d) < 1e-6:
            continue
        rays.append((o, d / np.linalg.norm(d)))
    return np.array(tris), rays


def _brute(tris, o, d, eps=1e-14):
    """Möller–Trumbore in f64 over every triangle (mesh.rs:117-142 rules)."""
    v0, v1, v2 = tris[:, 0], tris[:, 1], tris[:, 2]
    e1, e2 = v1 - v0, v2 - v0
    p = np.cross(d, e2)
    det = (e1 * p).sum(1)
    ok = np.abs(det) >= eps
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    tv = o - v0
    u = (tv * p).sum(1) * inv
    q = np.cross(tv, e1)
    v = (d * q).sum(1) * inv
    t = (e2 * q).sum(1) * inv
    hit = ok & (u >= 0) & (u <= 1) & (v >= 0) & (u + v <= 1) & (t > 1e-9)
    if not hit.any():
        return None, np.inf
    t = np.where(hit, t, np.inf)
    i = int(np.argmin(t))
    return i, t[i]


def test_bvh_matches_brute_force():
    """bvh.rs:403-453: BVH closest hit == brute force on prim id, t within 1e-9."""
    tris, rays = _lcg_soup()
    tris = tris.astype(np.float32).astype(np.float64)  # meshes store f32 positions
    s = scene.Scene(8, 8)
    s.add_instance(s.add_mesh(tris.reshape(-1, 3), np.arange(len(tris) * 3).reshape(-1, 3)),
                   s.add_material(scene.matte((0.5, 0.5, 0.5))))
    o_s = oracle.OracleScene(s)
    planes = np.zeros((2, len(rays), 4), dtype=np.float32)
    for k, (o, d) in enumerate(rays):
        planes[0, k, :3] = o
        planes[1, k, :3] = d
        planes[1, k, 3] = np.inf
    prim, inst, t, _ = o_s.intersect(planes, threads=1)
    for k, (o, d) in enumerate(rays):
        o32 = planes[0, k, :3].astype(np.float64)
        d32 = planes[1, k, :3].astype(np.float64)
        bi, bt = _brute(tris, o32, d32)
        if bi is None:
            assert prim[k] == 0xFFFFFFFF
        else:
            assert prim[k] == bi and abs(t[k] - bt) < 1e-9, (k, prim[k], bi, t[k], bt)


def test_any_hit_respects_limit():
    """bvh.rs:455-472: one triangle at z = 5; any hit within 10 yes, within 4 no."""
    s = scene.Scene(8, 8)
    s.add_instance(s.add_mesh([[-1, -1, 5], [1, -1, 5], [0, 1, 5]], [[0, 1, 2]]),
                   s.add_material(scene.matte((0.5, 0.5, 0.5))))
    o_s = oracle.OracleScene(s)
    planes = np.zeros((2, 2, 4), dtype=np.float32)
    planes[1, :, 2] = 1.0
    planes[1, 0, 3] = 10.0
    planes[1, 1, 3] = 4.0
    hit, _, _, _ = o_s.intersect(planes, any_hit=True)
    assert hit.tolist() == [1, 0]


def _cube_scene(xform):
    s = scene.Scene(8, 8)
    p, i = scenes.unit_cube()
    m = s.add_mesh(p * 2.0, i)   # the reference's test cube spans [-1, 1]^3
    s.add_instance(m, s.add_material(scene.matte((0.5, 0.5, 0.5))), xform)
    return s


def test_cube_instance_hits_at_4():
    """mesh.rs:473-488: unit cube translated to z = 5, ray from the origin: t = 4."""
    o_s = oracle.OracleScene(_cube_scene(scene.affine(None, (0, 0, 5))))
    planes = np.zeros((2, 1, 4), dtype=np.float32)
    planes[1, 0] = [0, 0, 1, np.inf]
    prim, inst, t, _ = o_s.intersect(planes)
    assert inst[0] == 0 and abs(t[0] - 4.0) < 1e-9


def test_scaled_instance_t_is_world():
    """mesh.rs:490-500: scale 2 then translate z = 5: front face at z = 3, t = 3."""
    o_s = oracle.OracleScene(_cube_scene(scene.affine(np.eye(3) * 2.0, (0, 0, 5))))
    planes = np.zeros((2, 1, 4), dtype=np.float32)
    planes[1, 0] = [0, 0, 1, np.inf]
    _, _, t, _ = o_s.intersect(planes)
    assert abs(t[0] - 3.0) < 1e-9


def _mat(**kw):
    m = abi.RtMaterialDesc()
    for k, v in kw.items():
        setattr(m, k, abi.c_double3(*v) if isinstance(v, tuple) else v)
    return m


def diffuse_params():
    """bxdf.rs:380-387 params_diffuse: gain 1, colour 1, specular_ior 1."""
    return _mat(**scene.matte((1.0, 1.0, 1.0)))


def metal_params(color, rough):
    return _mat(**scene.ggx_conductor(color, rough))


def plastic_params(color, rough):
    return _mat(**scene.ggx_floor(color, rough))


def test_pdf_integrates_to_one():
    """bxdf.rs:391-426: the composite pdf integrates to 1 +- 0.05 over the
    reflection hemisphere (64 x 128 midpoint grid, wo = (0.3,-0.15,0.94))."""
    cases = [diffuse_params(), metal_params((0.9, 0.7, 0.4), 0.3), plastic_params((0.5, 0.2, 0.2), 0.15)]
    wo = np.array([0.3, -0.15, 0.94])
    wo /= np.linalg.norm(wo)
    nt, npp = 64, 128
    for ci, m in enumerate(cases):
        total = 0.0
        for it in range(nt):
            th = (it + 0.5) / nt * (np.pi / 2)
            for ip in range(npp):
                ph = (ip + 0.5) / npp * 2 * np.pi
                wi = [np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)]
                _, pdf = oracle.bsdf_eval(m, wo, wi, 1.5)
                total += pdf * np.sin(th) * (np.pi / 2 / nt) * (2 * np.pi / npp)
        assert abs(total - 1.0) < 0.05, (ci, total)


def test_furnace_estimates():
    """bxdf.rs:428-453: diffuse 1 +- 0.02; metal <= 1.02 and > 0.75; plastic <= 1.03."""
    wo = np.array([0.2, 0.1, 0.97])
    wo /= np.linalg.norm(wo)
    d, _ = oracle.bsdf_furnace(diffuse_params(), wo, 1.5, 200_000)
    assert abs(d - 1.0) < 0.02
    m, _ = oracle.bsdf_furnace(metal_params((1, 1, 1), 0.4), wo, 1.5, 200_000)
    assert 0.75 < m <= 1.02
    p, _ = oracle.bsdf_furnace(plastic_params((1, 1, 1), 0.2), wo, 1.5, 200_000)
    assert p <= 1.03


def test_estimator_consistency():
    """bxdf.rs:455-487: BSDF-sampled and uniform-hemisphere estimates of the
    reflected energy agree within 3% (metal 0.8/0.6/0.3, roughness 0.35)."""
    m = metal_params((0.8, 0.6, 0.3), 0.35)
    wo = np.array([-0.3, 0.2, 0.93])
    wo /= np.linalg.norm(wo)
    by_bsdf, _ = oracle.bsdf_furnace(m, wo, 1.5, 400_000, seed=3, stream=9)
    u = oracle.pcg_new_stream(5, 17, 2 * 100_000).astype(np.float64) / 2.0 ** 32
    acc = 0.0
    for k in range(100_000):
        z = u[2 * k]
        r = np.sqrt(max(0.0, 1 - z * z))
        ph = 2 * np.pi * u[2 * k + 1]
        f, _ = oracle.bsdf_eval(m, wo, [r * np.cos(ph), r * np.sin(ph), z], 1.5)
        acc += (0.2126 * f[0] + 0.7152 * f[1] + 0.0722 * f[2]) * z * 2 * np.pi
    by_uniform = acc / 100_000
    assert abs(by_bsdf - by_uniform) / by_uniform < 0.03, (by_bsdf, by_uniform)


def _light_scene(lights):
    s = scene.Scene(8, 8)
    for kind, args in lights:
        getattr(s, kind)(*args)
    return s


def test_light_pmf_normalised_and_consistent():
    """light_sampler.rs:324-355: sum of pmf over all lights = 1 +- 1e-9 and
    sample()'s pmf equals pmf(). The reference mixes in a dome light; the
    infinite group here is a distant light (dome lights are out of scope)."""
    lights = []
    for i in range(40):
        a = i * 0.7
        lights.append(("add_point_light", ((np.cos(a) * (5 + i % 7), i % 5, np.sin(a) * (5 + (i % 3) * 3)),
                                           0.5 + i % 4)))
    lights.append(("add_distant_light", ((0, -1, 0), 0.5)))
    o_s = oracle.OracleScene(_light_scene(lights))
    p = [1.0, 0.5, -2.0]
    total = sum(o_s.light_pmf(p, i) for i in range(len(lights)))
    assert abs(total - 1.0) < 1e-9
    for k in range(200):
        li, pmf = o_s.light_sample(p, (k + 0.5) / 200)
        re = o_s.light_pmf(p, li)
        assert abs(pmf - re) < 1e-9 * max(pmf, re, 1e-12)


def test_light_importance_prefers_near():
    """light_sampler.rs:359-371: a near light's pmf > 0.25 among 64."""
    lights = [("add_point_light", ((0, 1, 0), 10.0))]
    lights += [("add_point_light", ((500.0 + i, 1, 500), 10.0)) for i in range(63)]
    o_s = oracle.OracleScene(_light_scene(lights))
    assert o_s.light_pmf([0, 0, 0.5], 0) > 0.25


@pytest.fixture(scope="module")
def cornell48():
    s = scenes.cornell_box(48, 48)
    return s, oracle.OracleScene(s)


def test_cornell_renders_with_gi(cornell48):
    """pt_tests.rs:16-54: the lit box is neither black nor blown out, the left
    third is red-dominant, the right third green-dominant, and the ceiling
    corner is lit indirectly."""
    s, o_s = cornell48
    rgb, _, _ = o_s.render(abi.make_params(max_depth=8), 0, 32)
    img = (rgb / 32).reshape(48, 48, 3)
    mean = img.reshape(-1, 3).mean(0)
    lum = 0.2126 * mean[0] + 0.7152 * mean[1] + 0.0722 * mean[2]
    assert 0.05 < lum < 2.0
    left = img[12:36, :16].reshape(-1, 3).mean(0)
    right = img[12:36, 32:].reshape(-1, 3).mean(0)
    assert left[0] > left[1] and right[1] > right[0]
    assert img[6, 6].sum() > 0.03


def test_oracle_deterministic(cornell48):
    """pt_tests.rs:56-69: same seed, bitwise identical output."""
    s, o_s = cornell48
    p = abi.make_params(max_depth=8)
    a, _, _ = o_s.render(p, 0, 4)
    b, _, _ = o_s.render(p, 0, 4, threads=3)
    assert np.array_equal(a, b)


def test_oracle_converges():
    """pt_tests.rs:71-95: RMSE at 64 spp < 0.6 x RMSE at 4 spp vs a 256-spp render."""
    s = scenes.cornell_box(16, 16)
    o_s = oracle.OracleScene(s)
    p = abi.make_params(max_depth=8)
    ref = o_s.render(p, 0, 256)[0] / 256
    coarse = o_s.render(p, 1000, 1004)[0] / 4
    fine = o_s.render(p, 2000, 2064)[0] / 64
    rmse = lambda x: np.sqrt(((x - ref) ** 2).mean())
    assert rmse(fine) < 0.6 * rmse(coarse)


def test_sample_ranges_add_up(cornell48):
    """render_sum (mod.rs:106-133): per-(pixel, sample) seeding makes sample
    ranges add up to the full render (f64 summation order aside)."""
    s, o_s = cornell48
    p = abi.make_params(max_depth=8)
    full = o_s.render(p, 0, 6)[0]
    parts = o_s.render(p, 0, 2)[0] + o_s.render(p, 2, 6)[0]
    assert np.allclose(full, parts, rtol=1e-12, atol=1e-12)


def test_constant_dome_furnace():
    # A convex Lambertian sphere of albedo rho inside a constant dome of
    # radiance 1: every surface point reflects rho * 1 (no interreflection),
    # and camera rays that miss see the dome itself (mod.rs:643-656, 1139-1172).
    from rtcuda import abi, scenes
    from rtcuda.scene import Scene, matte
    s = Scene(24, 24, fov=30.0)
    s.look_at((0, 0, -4.0), (0, 0, 0))
    pos, idx, nrm = scenes.icosphere(4)
    s.add_instance(s.add_mesh(pos, idx, normals=nrm), s.add_material(matte((0.5, 0.5, 0.5))))
    s.add_dome_light(1.0, (1.0, 1.0, 1.0))
    p = abi.make_params(max_depth=8)
    spp = 256
    img = oracle.OracleScene(s).render(p, 0, spp)[0].reshape(24, 24, 3) / spp
    np.testing.assert_allclose(img[0, 0], 1.0, rtol=1e-12)          # a miss: the dome
    centre = img[9:15, 9:15].mean((0, 1))
    np.testing.assert_allclose(centre, 0.5, rtol=0.03)


def _patch_map(w=32, h=16):
    m = np.full((h, w, 3), 0.05, np.float32)
    m[4:8, 10:16] = 5.0
    return m


def test_envmap_sample_pdf_consistency():
    # envmap.rs tests (sample_pdf_consistency): the pdf integrates to ~1 over
    # the sphere, samples land on the bright patch and carry its radiance.
    env = _patch_map()
    nt, npp = 128, 256
    th = (np.arange(nt) + 0.5) / nt * np.pi
    ph = (np.arange(npp) + 0.5) / npp * 2 * np.pi
    T, Ph = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(T) * np.sin(Ph), np.cos(T), -np.sin(T) * np.cos(Ph)], -1).reshape(-1, 3)
    _, pdf = oracle.env_eval_pdf(env, d)
    integral = float((pdf * np.sin(T).ravel()).sum() * (np.pi / nt) * (2 * np.pi / npp))
    assert abs(integral - 1.0) < 0.03, integral
    state = 0x1234
    uv = []
    for _ in range(400):
        state = (state * 6364136223846793005 + 1) % (1 << 64)
        uv.append((state >> 11) / float(1 << 53))
    dirs, rad, pdf = oracle.env_sample(env, np.array(uv).reshape(200, 2))
    assert (pdf > 0).all()
    rad2, _ = oracle.env_eval_pdf(env, dirs)
    np.testing.assert_allclose(rad2, rad, atol=1e-9)
    assert (rad[:, 0] > 1.0).sum() > 150


def test_uniform_envmap_equals_constant_dome():
    # A map of ones under intensity 1 is the constant dome of radiance 1:
    # same image in expectation (the sampling densities differ).
    from rtcuda.scene import Scene, matte
    pos, idx, nrm = scenes.icosphere(3)
    imgs = []
    for env in (None, np.ones((8, 16, 3), np.float32)):
        s = scene.Scene(16, 16, fov=30.0)
        s.look_at((0, 0, -4.0), (0, 0, 0))
        s.add_instance(s.add_mesh(pos, idx, normals=nrm), s.add_material(matte((0.5, 0.5, 0.5))))
        s.add_dome_light(1.0, (1.0, 1.0, 1.0), env=env)
        p = abi.make_params(max_depth=6)
        imgs.append(oracle.OracleScene(s).render(p, 0, 512)[0].reshape(16, 16, 3) / 512)
    np.testing.assert_allclose(imgs[0][0, 0], imgs[1][0, 0], rtol=1e-12)
    np.testing.assert_allclose(imgs[0][6:10, 6:10].mean(), imgs[1][6:10, 6:10].mean(), rtol=0.03)


@pytest.mark.parametrize("kind,width", [(abi.FILTER_BOX, 1.0), (abi.FILTER_TRIANGLE, 2.0), (abi.FILTER_GAUSSIAN, 2.0)])
def test_filter_samples_stay_in_support_and_center(kind, width):
    """camera.rs:213-239: 4096 stratified uniforms; every offset within half
    the width, mean offset below 0.05."""
    u = (np.arange(4096) + 0.5) / 4096
    dx = oracle.filter_sample(kind, width, u)
    assert np.all(np.abs(dx) <= width * 0.5 + 1e-9)
    assert abs(dx.mean()) < 0.05, dx.mean()


def test_gaussian_second_uniform_needs_f64():
    """The Gaussian filter's second uniform fract(u * 2654435761)
    (camera.rs:55) collapses to 0 when the product is rounded to f32, which
    would fail the centring test above: why the CUDA raygen forms it in f64."""
    u = ((np.arange(4096) + 0.5) / 4096).astype(np.float32)
    x32 = u * np.float32(2654435761.0)
    assert np.mean(x32 - np.trunc(x32) == 0) > 0.99
    x64 = u.astype(np.float64) * 2654435761.0
    u2 = x64 - np.trunc(x64)
    g = np.sqrt(-2.0 * np.log(np.maximum(u.astype(np.float64), 1e-12))) * np.cos(2.0 * np.pi * u2)
    np.testing.assert_allclose(np.clip(g * 0.5, -1.0, 1.0), oracle.filter_sample(abi.FILTER_GAUSSIAN, 2.0, u),
                               atol=1e-6)
