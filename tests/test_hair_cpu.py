"""Curves and Marschner hair in the f64 oracle, pinned by the reference's
own unit tests (src/geometry/curves.rs:249-345, src/raytracer/pt/hair.rs:
413-473) and scene-level checks of curve instances."""
import numpy as np

import oracle
from rtcuda import abi, scene


def test_capsule_hit_and_normal():
    """curves.rs:254-276."""
    out = oracle.curve_segment((-1, 0, 0, 0.5), (1, 0, 0, 0.5), 0.0, 1.0,
                               [(0.2, 0, -5), (1.4, 0, -5), (0, 2, -5)], [(0, 0, 1)] * 3)
    t, n, tang, v = out[0, 0], out[0, 1:4], out[0, 4:7], out[0, 7]
    assert abs(t - 4.5) < 1e-9 and n[2] < -0.99 and abs(tang[0]) > 0.99 and 0.5 < v < 0.7
    assert out[1, 0] > 0 and out[1, 1] > 0.3   # cap hit past the end
    assert out[2, 0] < 0                         # clean miss


def test_tapered_cone_radius():
    """curves.rs:278-290: radius 0.5 -> 0.1, surface near y ~ 0.3 at x = 0."""
    out = oracle.curve_segment((-1, 0, 0, 0.5), (1, 0, 0, 0.1), 0.0, 1.0, [(0, 5, 0)], [(0, -1, 0)])
    y = 5.0 - out[0, 0]
    assert 0.25 < y < 0.36


def test_point_particle_is_sphere():
    """curves.rs:322-334."""
    out = oracle.curve_segment((0, 0, 5, 0.25), (0, 0, 5, 0.25), 0.0, 1.0, [(0, 0, 0)], [(0, 0, 1)])
    assert abs(out[0, 0] - 4.75) < 1e-9 and out[0, 3] < -0.99


HAIR = ((0.0, 0.0, 0.0), 0.3, 0.3, 1.55)


def test_hair_white_furnace():
    """hair.rs:419-442: with zero absorption the fiber scatters all energy,
    the integral of f over the sphere is 1 for any wo and h."""
    rng = np.random.default_rng(7)
    for sin_to, h in ((0.0, 0.0), (0.4, 0.3), (-0.7, -0.6), (0.2, 0.9)):
        wo = np.array([sin_to, np.sqrt(1 - sin_to ** 2), 0.0])
        u1, u2 = rng.random(40_000), rng.random(40_000)
        z = 1 - 2 * u1
        r = np.sqrt(np.maximum(1 - z * z, 0))
        wi = np.stack([z, r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)], axis=1)
        f, _ = oracle.hair_eval(HAIR, wo, wi, h)
        mean = (f * 4 * np.pi).mean(0)
        assert abs(mean[0] - 1.0) < 0.05, (sin_to, h, mean)


def test_hair_sampling_consistency():
    """hair.rs:444-461: E[f / pdf] over hair::sample equals the furnace
    integral, stream (pixel 11, sample 5); and the returned pdf is pdf()."""
    params = ((0.0, 0.0, 0.0), 0.35, 0.4, 1.55)
    wo = np.array([0.3, np.sqrt(1 - 0.09), 0.0])
    wi, f, pdf = oracle.hair_sample(params, wo, -0.4, 11, 5, 40_000)
    ok = pdf > 0
    lum = 0.2126 * f[:, 0] + 0.7152 * f[:, 1] + 0.0722 * f[:, 2]
    assert abs((lum[ok] / pdf[ok]).sum() / len(pdf) - 1.0) < 0.05
    f2, p2 = oracle.hair_eval(params, wo, wi[ok][:500], -0.4)
    np.testing.assert_allclose(p2, pdf[ok][:500], rtol=1e-12)
    np.testing.assert_allclose(f2, f[ok][:500], rtol=1e-12)


def test_hair_absorption_darkens():
    """hair.rs:463-474: absorption darkens the transmission lobe."""
    wo, wi = np.array([0.0, 1.0, 0.0]), np.array([0.0, -1.0, 0.0])
    fw, _ = oracle.hair_eval(HAIR, wo, wi, 0.0)
    fd, _ = oracle.hair_eval(((3.0, 3.0, 3.0), 0.3, 0.3, 1.55), wo, wi, 0.0)
    assert fd[0, 0] < fw[0, 0] * 0.2


def test_fiber_frame_h_spans_width():
    """hair.rs:476-486."""
    t, wo = (1, 0, 0), (0, 0, 1)
    assert abs(oracle.fiber_h(t, (0, 0, 1), wo)) < 1e-9
    assert abs(oracle.fiber_h(t, (0, 1, 0), wo)) > 0.99


def test_sigma_a_from_color():
    """hair.rs:61-76 (pbrt's SigmaAFromReflectance) through the scene helper."""
    m = scene.marschner_hair(color=(0.5, 0.3, 0.1), azimuthal_roughness=0.3)
    bn = 0.3
    den = 5.969 - 0.215 * bn + 2.532 * bn ** 2 - 10.73 * bn ** 3 + 5.574 * bn ** 4 + 0.245 * bn ** 5
    np.testing.assert_allclose(m["hair_sigma_a"], (np.log([0.5, 0.3, 0.1]) / den) ** 2, rtol=1e-12)


def _hair_scene(w=16, h=16):
    s = scene.Scene(w, h, fov=30.0)
    s.look_at((0.0, 0.0, 4.0), (0.0, 0.0, 0.0))
    # A comb of 40 vertical strands, each 8 segments with a taper.
    p0, p1, v0, v1 = [], [], [], []
    for k in range(40):
        x = -0.8 + 1.6 * k / 39
        for j in range(8):
            y0, y1 = -1 + 2 * j / 8, -1 + 2 * (j + 1) / 8
            r0, r1 = 0.02 * (1 - j / 8) + 0.005, 0.02 * (1 - (j + 1) / 8) + 0.005
            p0.append((x + 0.05 * np.sin(3 * y0), y0, 0.1 * np.cos(2 * x), r0))
            p1.append((x + 0.05 * np.sin(3 * y1), y1, 0.1 * np.cos(2 * x), r1))
            v0.append(j / 8)
            v1.append((j + 1) / 8)
    cs = s.add_curves(p0, p1, v0, v1)
    hm = s.add_material(scene.marschner_hair(color=(0.6, 0.4, 0.2)))
    s.add_instance(cs, hm)
    s.add_rect_light((-1, 2, 1), (2, 0, 0), (0, 0, 1), 10.0)
    s.background = (0.05, 0.05, 0.08)
    return s


def test_curve_instance_hits_and_tangent():
    """Rays into the comb meet the strands through the curve instance."""
    s = _hair_scene()
    o = oracle.OracleScene(s)
    planes = np.zeros((2, 3, 4), np.float32)
    planes[0, :, :3] = [(-0.8, 0.0, 4.0), (0.0, 0.0, 4.0), (0.9, 0.0, 4.0)]
    planes[1, :, :3] = (0, 0, -1)
    planes[1, :, 3] = np.inf
    prim, inst, t, _ = o.intersect(planes)
    assert inst[0] == 0 and 3.8 < t[0] < 4.0      # the first strand
    assert inst[2] == 0xFFFFFFFF                  # beyond the comb


def test_hair_render_is_lit():
    """The oracle renders the comb under the rect light: finite and lit."""
    s = _hair_scene()
    img = oracle.OracleScene(s).render(abi.make_params(max_depth=8), 0, 16)[0] / 16
    assert np.isfinite(img).all() and img.mean() > 0.01


def test_dice_bezier_curve():
    """curves.rs:292-320: one cubic Bezier span diced into 8 segments."""
    from rtcuda.patches import BASES
    from rtcuda.rib import dice_curve
    p0, p1, v0, v1 = dice_curve([[0, 0, 0], [0, 1, 0], [1, 2, 0], [2, 2, 0]], (BASES["bezier"][0], 3), 0.1, 0.02, 8)
    assert len(p0) == 8
    assert abs(p0[0][0]) < 1e-6 and abs(p0[0][1]) < 1e-6
    assert abs(p1[7][0] - 2.0) < 1e-6 and abs(p1[7][1] - 2.0) < 1e-6
    assert p0[0][3] > p1[7][3] and abs(p0[0][3] - 0.05) < 1e-6
    assert v0[0] == 0.0 and v1[7] == 1.0


def test_rib_curves_points_and_hair():
    """Curves / Points requests (scene_builder.rs:1050-1170) with a
    PxrMarschnerHair material (hair.rs:82-100)."""
    from rtcuda.rib import load_rib_string
    s = load_rib_string("""
Format 8 8 1
WorldBegin
  Bxdf "PxrMarschnerHair" "h" "roughness" [0.25] "azimuthalRoughness" [0.4] "color" [0.5 0.3 0.1]
  Curves "cubic" [4 4] "nonperiodic" "P" [0 0 0 0 1 0 1 2 0 2 2 0  0 0 1 0 1 1 1 2 1 2 2 1] "width" [0.1 0.02]
  Bxdf "PxrSurface" "s" "diffuseColor" [0.5 0.5 0.5]
  Curves "linear" [3] "nonperiodic" "P" [0 0 0 1 0 0 2 0 0] "constantwidth" [0.04]
  Points "P" [0 0 5 1 0 5] "width" [0.2 0.4]
WorldEnd
""")
    assert len(s.curves) == 3
    p0, p1, v0, v1 = s.curves[0]
    assert len(p0) == 2 * 8  # two cubic Bezier curves, 8 segments each at shading rate 1
    hair = s.materials[s.instance_array()["mat"][0]]
    assert hair["hair"] == 1 and hair["hair_beta_m"] == 0.25 and hair["hair_beta_n"] == 0.4
    lin = s.curves[1]
    assert len(lin[0]) == 2 and abs(lin[0][0][3] - 0.02) < 1e-7
    pts = s.curves[2]
    assert np.array_equal(pts[0], pts[1]) and abs(pts[0][1][3] - 0.2) < 1e-7 and (pts[2] == 0.5).all()
    assert s.materials[s.instance_array()["mat"][1]]["hair"] == 0
