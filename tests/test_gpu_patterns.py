"""Procedural patterns on the GPU (csrc/pattern.cuh) against the f64
oracle's restatement of src/texture/pattern.rs and shade_params
(pt/mod.rs:389-439): the same scene through both, statistical parity as
in the other render tests, the ray-cone footprint filtering a checker
finer than a pixel to its mean colour, and cutouts whose presence is a
pattern (decided in shading and at every shadow-ray blocker,
pt/mod.rs:1244-1306, kernel_pt.metal:1336-1378)."""
import numpy as np
import pytest

import oracle
from mc_parity import compare, render_quad
from rtcuda import PtSession, abi, scene, scenes

pytestmark = pytest.mark.gpu


def _render(s, p, spp):
    with PtSession(s, p) as g:
        g.render_samples(0, spp)
        return g.image()


def test_patterned_room_matches_oracle():
    w, h, spp = 96, 72, 256
    p = abi.make_params(max_depth=6)
    s = scenes.patterned_room(w, h)
    gpu = _render(s, p, spp)
    cpu = oracle.OracleScene(s).render(p, 0, spp)[0].reshape(h, w, 3) / spp
    plain = scenes.patterned_room(w, h)
    plain.bindings = []
    flat = oracle.OracleScene(plain).render(p, 0, spp)[0].reshape(h, w, 3) / spp
    np.testing.assert_allclose(gpu.mean((0, 1)), cpu.mean((0, 1)), rtol=0.03)
    for axis in (0, 1):
        a, b = gpu.mean(axis).mean(-1), cpu.mean(axis).mean(-1)
        assert np.all(np.abs(a - b) <= 0.08 * b + 0.015), (axis, np.abs(a - b).max())
    same, other = np.abs(gpu - cpu).mean(), np.abs(gpu - flat).mean()
    assert same < 0.5 * other, (same, other)


def _fine_checker_plane(fine):
    s = scene.Scene(48, 32, fov=40.0)
    s.look_at((0.0, 1.5, -3.0), (0.0, 0.0, 1.0))
    if fine:
        m = s.add_material(scene.matte((1.0, 1.0, 1.0)))
        s.bind_pattern(m, "diffuseColor", s.add_checker((0.9, 0.5, 0.1), (0.1, 0.3, 0.7), scale=(512.0, 512.0)))
    else:
        m = s.add_material(scene.matte((0.5, 0.4, 0.4)))
    plane = s.add_mesh([[-2, 0, -2], [2, 0, -2], [2, 0, 2], [-2, 0, 2]], [[0, 2, 1], [0, 3, 2]],
                       st=[[0, 0], [1, 0], [1, 1], [0, 1]])
    s.add_instance(plane, m)
    s.add_distant_light((0.3, -1.0, 0.2), 2.0)
    return s


def test_footprint_filters_a_sub_pixel_checker_to_its_mean():
    # Cells of 1/512 st (1/128 world units) against a footprint of at least
    # ~1/250 st at every hit: the blend weight saturates at 1, so the
    # checker shades as its mean colour, the same material as the plain one.
    p = abi.make_params(max_depth=3)
    fine, flat = _render(_fine_checker_plane(True), p, 16), _render(_fine_checker_plane(False), p, 16)
    assert flat.mean() > 0.05
    np.testing.assert_allclose(fine, flat, rtol=1e-4, atol=1e-5)


def _textured_scene(w=64, h=48, bind=True):
    """A floor with an st-mapped texture (the EWA path: mesh st and a ray
    cone) and a block with a triplanar projection of the same texture."""
    s = scene.Scene(w, h, fov=45.0)
    s.look_at((0.0, 1.3, -2.6), (0.0, 0.2, 1.0))
    x, y = np.meshgrid(np.arange(64), np.arange(64))
    cells = ((x // 8 + y // 8) % 2).astype(np.float32)
    img = np.stack([0.15 + 0.7 * cells, 0.2 + 0.6 * x / 63.0, 0.8 - 0.6 * y / 63.0], -1).astype(np.float32)
    t = s.add_texture(img)
    floor_m = s.add_material(scene.matte((0.5, 0.5, 0.5)))
    block_m = s.add_material(scene.ggx_floor((0.5, 0.5, 0.5), 0.4))
    if bind:
        s.bind_pattern(floor_m, "diffuseColor", s.add_texture_node(t, scale=(3.0, 3.0)))
        s.bind_pattern(block_m, "diffuseColor", s.add_triplanar(t, wrap="periodic", frequency=1.5))
    plane = s.add_mesh([[-3, 0, -2], [3, 0, -2], [3, 0, 4], [-3, 0, 4]], [[0, 2, 1], [0, 3, 2]],
                       st=[[0, 0], [1, 0], [1, 1], [0, 1]])
    s.add_instance(plane, floor_m)
    from rtcuda.scenes import unit_cube
    cp, ci = unit_cube()
    s.add_instance(s.add_mesh(cp, ci), block_m, scene.affine(scene.rot_y(30) * 0.6, (0.5, 0.3, 1.2)))
    s.add_distant_light((0.4, -1.0, 0.3), 2.5)
    s.add_point_light((-1.0, 2.0, 0.0), 3.0)
    return s


def test_textures_match_oracle():
    w, h, spp = 64, 48, 256
    p = abi.make_params(max_depth=5, aovs=True)
    s = _textured_scene(w, h)
    with PtSession(s, p) as g:
        g.render_samples(0, spp)
        gpu, gaux = g.image(), g.aux()
    rgb, aux, _ = oracle.OracleScene(s).render(p, 0, spp, aovs=True)
    cpu, caux = rgb.reshape(h, w, 3) / spp, aux.reshape(h, w, 12)
    # First-hit albedo: the texture lookups themselves (no transport noise;
    # only sub-pixel positions differ between the two samplers).
    ga, ca = gaux[..., 0:3] / spp, caux[..., 0:3] / spp
    assert np.abs(ga - ca).mean() < 0.004, np.abs(ga - ca).mean()
    assert np.abs(ga - ca).max() < 0.08, np.abs(ga - ca).max()
    flat = _textured_scene(w, h, bind=False)
    fa = oracle.OracleScene(flat).render(p, 0, 16, aovs=True)[1].reshape(h, w, 12)[..., 0:3] / 16
    assert np.abs(fa - ca).mean() > 10 * np.abs(ga - ca).mean()
    np.testing.assert_allclose(gpu.mean((0, 1)), cpu.mean((0, 1)), rtol=0.03)
    for axis in (0, 1):
        a, b = gpu.mean(axis).mean(-1), cpu.mean(axis).mean(-1)
        assert np.all(np.abs(a - b) <= 0.08 * b + 0.015), (axis, np.abs(a - b).max())


def test_ies_point_light_matches_oracle():
    """A narrow downlight profile (src/scene/ies.rs) on a point light above a
    floor, tilted 30 degrees: GPU against the oracle, and unlike the bare light."""
    from rtcuda.ies import parse_ies
    from test_ies_cpu import DOWNLIGHT
    w, h, spp = 48, 36, 64

    def make(profile):
        s = scene.Scene(w, h, fov=60.0)
        s.look_at((0.0, 2.5, -2.5), (0.0, 0.0, 0.5))
        m = s.add_material(scene.matte((0.7, 0.7, 0.7)))
        s.add_instance(s.add_mesh([[-4, 0, -3], [4, 0, -3], [4, 0, 5], [-4, 0, 5]], [[0, 2, 1], [0, 3, 2]]), m)
        a = np.radians(30.0)
        tilt = np.array([[1, 0, 0], [0, np.cos(a), -np.sin(a)], [0, np.sin(a), np.cos(a)]])
        s.add_point_light((0.0, 1.5, 0.5), 6.0, ies=parse_ies(DOWNLIGHT) if profile else None,
                          world_to_local=tilt.T)
        return s

    p = abi.make_params(max_depth=3)
    s = make(True)
    gpu = _render(s, p, spp)
    cpu = oracle.OracleScene(s).render(p, 0, spp)[0].reshape(h, w, 3) / spp
    bare = oracle.OracleScene(make(False)).render(p, 0, spp)[0].reshape(h, w, 3) / spp
    np.testing.assert_allclose(gpu.mean((0, 1)), cpu.mean((0, 1)), rtol=0.03)
    same, other = np.abs(gpu - cpu).mean(), np.abs(gpu - bare).mean()
    assert same < 0.2 * other, (same, other)


def test_udim_tiles_match_oracle():
    """A floor whose st spans 2 x 2 UDIM cells, one constant-colour texture
    per tile: the GPU's first-hit albedo equals the oracle's."""
    w, h, spp = 32, 24, 64
    s = scene.Scene(w, h, fov=50.0)
    s.look_at((0.0, 2.0, -2.0), (0.0, 0.0, 0.3))
    colors = {1001: (0.9, 0.1, 0.1), 1002: (0.1, 0.9, 0.1), 1011: (0.1, 0.1, 0.9), 1012: (0.9, 0.9, 0.1)}
    tiles = {t: s.add_texture(np.tile(np.array(c, np.float32), (8, 8, 1))) for t, c in colors.items()}
    m = s.add_material(scene.matte((0.5, 0.5, 0.5)))
    s.bind_pattern(m, "diffuseColor", s.add_texture_node(-1, udim=tiles))
    s.add_instance(s.add_mesh([[-2, 0, -1], [2, 0, -1], [2, 0, 3], [-2, 0, 3]], [[0, 2, 1], [0, 3, 2]],
                              st=[[0, 0], [2, 0], [2, 2], [0, 2]]), m)
    s.add_distant_light((0.2, -1.0, 0.1), 2.0)
    p = abi.make_params(max_depth=2, aovs=True)
    with PtSession(s, p) as g:
        g.render_samples(0, spp)
        ga = g.aux()[..., 0:3] / spp
    ca = oracle.OracleScene(s).render(p, 0, spp, aovs=True)[1].reshape(h, w, 12)[..., 0:3] / spp
    assert np.abs(ga - ca).mean() < 0.01, np.abs(ga - ca).mean()
    assert len(np.unique(np.round(ca.reshape(-1, 3), 1), axis=0)) >= 4


def test_pattern_cutouts_match_oracle():
    s = scenes.pattern_cutouts(48, 36)
    g, o, r, pr, st = render_quad(s, abi.make_params(max_depth=6), 32, 1024)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res


def test_pattern_cutouts_change_the_image():
    """The same screens without their presence patterns (solid) render
    differently: light and view pass through the holes."""
    s = scenes.pattern_cutouts(48, 36)
    with PtSession(s, abi.make_params(max_depth=6)) as g:
        g.render_samples(0, 256)
        img = g.image()
    flat = scenes.pattern_cutouts(48, 36)
    flat.bindings = [b for b in flat.bindings if b[1] != abi.FIELD_PRESENCE]
    with PtSession(flat, abi.make_params(max_depth=6)) as g:
        g.render_samples(0, 256)
        solid = g.image()
    assert abs(img.mean() - solid.mean()) > 0.02 * solid.mean()
