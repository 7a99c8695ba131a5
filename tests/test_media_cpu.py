"""Participating media and subsurface scattering in the f64 oracle, pinned by
the reference's own unit tests (src/scene/medium.rs:105-170,
src/raytracer/pt/volume.rs:279-365) and by closed forms of whole renders."""
import numpy as np

import oracle
from rtcuda import abi, scene


def _fog(sigma_s, sigma_a, **kw):
    return scene.medium((sigma_a,) * 3, (sigma_s,) * 3, **kw)


def test_hg_normalizes():
    """medium.rs:109-128: the phase integrates to 1 over the sphere."""
    rng = np.random.default_rng(0x12345678)
    z = 1.0 - 2.0 * rng.random(100_000)
    for g in (-0.6, 0.0, 0.3, 0.8):
        mean = (oracle.hg_phase(g, z) * 4.0 * np.pi).mean()
        assert abs(mean - 1.0) < 0.02, (g, mean)


def test_hg_sample_matches_pdf():
    """medium.rs:130-149: phase / pdf of sampled directions averages to 1,
    and the pdf is the phase of the sampled direction."""
    rng = np.random.default_rng(99)
    wo = np.array([0.0, 0.0, 1.0])
    for g in (0.0, 0.5, -0.4):
        s = oracle.hg_sample(g, wo, rng.random((50_000, 2)))
        cos = -(s[:, :3] @ wo)
        val = oracle.hg_phase(g, cos)
        assert abs((val / np.maximum(s[:, 3], 1e-12)).mean() - 1.0) < 0.01
        np.testing.assert_allclose(s[:, 3], val, rtol=1e-12)
        np.testing.assert_allclose(np.linalg.norm(s[:, :3], axis=1), 1.0, atol=1e-12)


def test_fbm_density_bounded():
    """medium.rs:151-169."""
    m = _fog(1.0, 0.1, g=0.4, fbm=dict(frequency=0.5, octaves=4, gain=0.5, lacunarity=2.0, coverage=0.55,
                                       sharpness=4.0))
    i = np.arange(500)
    pts = np.stack([i * 0.37, (i % 17) * 0.9, (i % 5) * 1.0], axis=1)
    d = oracle.medium_density(m, pts)
    assert ((d >= 0.0) & (d <= 1.0)).all()
    assert 0.0 < d.mean() < 1.0


def test_homogeneous_estimator_unbiased():
    """volume.rs:296-320: E[pass weight] = T(t_max) and the scatter weights
    integrate to sigma_s / sigma_t (1 - T), same stream (pixel 3, sample 7)."""
    m = _fog(0.6, 0.4)
    n = 200_000
    ps, ss, _ = oracle.medium_sample(m, (0, 0, 0), (0, 0, 1), 1.3, (1, 1, 1), 3, 7, n)
    expected_pass = np.exp(-1.3)
    assert abs(ps[0] / n - expected_pass) < 0.01
    assert abs(ss[0] / n - 0.6 * (1.0 - expected_pass)) < 0.01


def test_chromatic_homogeneous_estimator_unbiased():
    """The spectral one-sample MIS (volume.rs:51-105) stays unbiased per
    channel when the extinction differs per channel and beta is coloured."""
    m = scene.medium((0.1, 0.5, 1.5), (0.9, 0.5, 0.2))
    n = 400_000
    ps, ss, _ = oracle.medium_sample(m, (0, 0, 0), (0, 0, 1), 1.1, (1.0, 0.4, 0.1), 5, 2, n)
    st = np.array([1.0, 1.0, 1.7])
    T = np.exp(-st * 1.1)
    np.testing.assert_allclose(ps / n, T, atol=0.01)
    np.testing.assert_allclose(ss / n, np.array([0.9, 0.5, 0.2]) / st * (1 - T), atol=0.01)


def test_ratio_tracking_matches_quadrature():
    """volume.rs:322-364: ratio-tracked transmittance of an fBm medium
    against a Riemann sum of its optical depth (stream pixel 11, sample 4)."""
    m = _fog(0.7, 0.3, fbm=dict(frequency=0.8, octaves=3, gain=0.5, lacunarity=2.0, coverage=0.6, sharpness=3.0))
    origin = np.array([0.3, 0.2, -1.0])
    d = np.array([0.2, 0.1, 1.0])
    d /= np.linalg.norm(d)
    dist, steps = 4.0, 20_000
    t = (np.arange(steps) + 0.5) / steps * dist
    tau = oracle.medium_density(m, origin + t[:, None] * d).sum() * (dist / steps)
    mean = oracle.medium_transmittance(m, origin, d, dist, 11, 4, 30_000)
    assert abs(mean[0] - np.exp(-tau)) < 0.02


def test_delta_tracking_matches_ratio_tracking():
    """Delta tracking's pass weights and ratio tracking estimate the same
    transmittance of an fBm medium."""
    m = _fog(0.0, 1.0, fbm=dict(frequency=0.8, octaves=3, gain=0.5, lacunarity=2.0, coverage=0.6, sharpness=3.0))
    o, d = (0.3, 0.2, -1.0), (0.0, 0.0, 1.0)
    n = 100_000
    ps, ss, k = oracle.medium_sample(m, o, d, 3.0, (1, 1, 1), 1, 1, n)
    tr = oracle.medium_transmittance(m, o, d, 3.0, 2, 2, n)
    assert abs(ps[0] / n - tr[0]) < 0.01
    assert (ss == 0).all()  # sigma_s = 0: scatters carry no weight


def test_sss_medium_fits():
    """volume.rs:259-288: the albedo inversion and the Burley scaling."""
    color, dmfp = np.array([0.8, 0.5, 0.2]), np.array([0.5, 0.25, 0.1])
    sa, ss = oracle.sss_medium(color, dmfp)
    alpha = 1 - np.exp(-color * (11.43 - 15.38 * color + 13.91 * color ** 2))
    st = (1.85 - color + 7 * np.abs(color - 0.8) ** 3) / dmfp
    np.testing.assert_allclose(ss, alpha * st, rtol=1e-12)
    np.testing.assert_allclose(sa + ss, st, rtol=1e-12)


def _slab_scene(med, bg=(1.0, 0.5, 0.25)):
    s = scene.Scene(4, 4, fov=10.0)
    s.add_material(scene.matte((0.5,) * 3))
    s.background = bg
    s.add_medium(med, atmosphere=True)
    return s


def test_absorbing_atmosphere_attenuates_background():
    """Camera rays through an absorbing slab atmosphere (max_distance 2):
    the background arrives scaled by exp(-sigma_a * 2) per channel."""
    med = scene.medium((0.2, 0.5, 1.0), (0.0, 0.0, 0.0), max_distance=2.0)
    s = _slab_scene(med)
    # Pass weight T / pdf with pdf = mean_c T_c: 0.5% noise at 32,768 samples.
    img = oracle.OracleScene(s).render(abi.make_params(max_depth=4), 0, 2048)[0].reshape(-1, 3) / 2048
    want = np.array([1.0, 0.5, 0.25]) * np.exp(-np.array([0.2, 0.5, 1.0]) * 2.0)
    np.testing.assert_allclose(img.mean(0), want, rtol=0.03)


def test_scattering_atmosphere_conserves_energy():
    """A purely scattering, isotropic atmosphere lit only by a uniform white
    background: every path leaves with radiance 1 (it either passes or
    scatters losslessly), so the image is 1 everywhere up to roulette noise."""
    med = scene.medium((0.0, 0.0, 0.0), (0.7, 0.7, 0.7), g=0.3, max_distance=3.0)
    s = _slab_scene(med, bg=(1.0, 1.0, 1.0))
    img = oracle.OracleScene(s).render(abi.make_params(max_depth=10), 0, 512)[0].reshape(-1, 3) / 512
    np.testing.assert_allclose(img.mean(), 1.0, atol=0.03)


def test_volume_hull_toggles_medium():
    """An invisible hull sphere with an absorbing interior: rays through
    its centre lose exp(-sigma_a * 2r); rays that miss it see the
    background unchanged."""
    s = scene.Scene(8, 8, fov=30.0)
    s.background = (1.0, 1.0, 1.0)
    mi = s.add_medium(scene.medium((0.5, 0.5, 0.5), (0.0, 0.0, 0.0)))
    hull = s.add_material(scene.volume_hull(interior=mi))
    s.add_quadric(abi.QUADRIC_SPHERE, [1.0, -1.0, 1.0, 360.0], hull, scene.affine(np.eye(3), (0, 0, 10)))
    o = oracle.OracleScene(s)
    img = o.render(abi.make_params(max_depth=4), 0, 64)[0].reshape(8, 8, 3) / 64
    # The centre pixels look through ~2 units of medium; the corners miss.
    assert abs(img[0, 0, 0] - 1.0) < 1e-12
    centre = img[3:5, 3:5, 0].mean()
    assert 0.35 < centre < 0.45, centre  # exp(-1) = 0.37 on the axis, a little more off axis
