"""Procedural patterns on the GPU (csrc/pattern.cuh) against the f64
oracle's restatement of src/texture/pattern.rs and shade_params
(pt/mod.rs:389-439): the same scene through both, statistical parity as
in the other render tests, and the ray-cone footprint filtering a checker
finer than a pixel to its mean colour."""
import numpy as np
import pytest

import oracle
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
