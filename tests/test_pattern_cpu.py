"""Procedural patterns on the CPU: the f64 oracle pinned by the
reference's own pattern, noise and st tests (src/texture/pattern.rs:
310-373, src/geometry/displace.rs:130-144, src/geometry/mesh.rs:497-517),
and the pattern-graph checks the CUDA backend makes on the host when a
session is created."""
import ctypes as C

import numpy as np
import pytest

import oracle
from rtcuda import abi, backend, scene, scenes


def ctx(st, footprint=0.0, p=(0.0, 0.0, 0.0)):
    return [st[0], st[1], p[0], p[1], p[2], footprint]


def test_checker_mix_ramp_chain():
    """pattern.rs:310-350."""
    s = scene.Scene(4, 4)
    checker = s.add_checker((1, 0, 0), (0, 1, 0), scale=(2, 2))
    mix = s.add_mix(checker, (0, 0, 1), (0.5, 0, 0))
    ramp = s.add_ramp([0.0, 1.0], [[0, 0, 0], [1, 1, 1]])
    c = oracle.pattern_eval(s, checker, [ctx((0.25, 0.25)), ctx((0.75, 0.25))])
    assert abs(c[0, 0] - 1.0) < 1e-9 and abs(c[0, 1]) < 1e-9
    assert abs(c[1, 1] - 1.0) < 1e-9
    m = oracle.pattern_eval(s, mix, [ctx((0.25, 0.25))])[0]
    assert abs(m[0] - 0.5) < 1e-9 and abs(m[2] - 0.5) < 1e-9
    r = oracle.pattern_eval(s, ramp, [ctx((0.5, 0.0))])[0]
    assert abs(r[0] - 0.5) < 1e-9
    f = oracle.pattern_eval(s, checker, [ctx((0.25, 0.25), footprint=0.5)])[0]
    assert f[0] < 1.0 and f[1] > 0.0


def test_colorcorrect_gamma_and_saturation():
    """pattern.rs:352-366."""
    s = scene.Scene(4, 4)
    n = s.add_color_correct((0.25, 0.25, 0.25), gamma=2.0, saturation=0.0)
    c = oracle.pattern_eval(s, n, [ctx((0.0, 0.0))])[0]
    assert abs(c[0] - 0.5) < 1e-9 and abs(c[1] - 0.5) < 1e-9


def test_perlin_is_bounded_and_zero_at_lattice():
    """displace.rs:130-144, through a one-octave fractal node
    (value = perlin * 0.5 + 0.5)."""
    s = scene.Scene(4, 4)
    f = s.add_fractal(frequency=1.0, octaves=1)
    lattice = [ctx((0, 0), p=(i, j, 0.0)) for i in range(-3, 3) for j in range(-3, 3)]
    v = oracle.pattern_eval(s, f, lattice)
    assert np.abs(v - 0.5).max() < 1e-12
    t = np.arange(1000) * 0.113
    line = [ctx((0, 0), p=(x, x * 0.7 + 0.3, x * 1.3 + 0.9)) for x in t]
    noise = np.abs(oracle.pattern_eval(s, f, line)[:, 0] * 2.0 - 1.0).max()
    assert 0.05 < noise <= 1.3


def test_st_density_follows_instance_scale():
    """mesh.rs:497-517: a unit st quad scaled 2x has st (0.25, 0.5) and
    density 0.5 where the ray (0.5, 1, -3) +z meets it."""
    s = scene.Scene(4, 4)
    m = s.add_mesh([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], [[0, 1, 2], [0, 2, 3]],
                   st=[[0, 0], [1, 0], [1, 1], [0, 1]])
    s.add_instance(m, s.add_material(scene.matte((0.5, 0.5, 0.5))), scene.affine(np.eye(3) * 2.0))
    hit = oracle.OracleScene(s).intersect_st([[0.5, 1.0, -3.0]], [[0.0, 0.0, 1.0]])[0]
    assert hit[0] > 0
    np.testing.assert_allclose(hit[1:], [0.25, 0.5, 0.5], atol=1e-6)


def test_patterns_change_the_oracle_render():
    s = scenes.patterned_room(24, 18)
    p = abi.make_params(max_depth=4)
    a = oracle.OracleScene(s).render(p, 0, 16)[0]
    s.bindings = []
    s._desc = None
    b = oracle.OracleScene(s).render(p, 0, 16)[0]
    assert np.abs(a - b).mean() > 0.05 * np.abs(b).mean()


def _create(s, **kw):
    h = C.c_void_p()
    d = s.desc()
    p = abi.make_params(bvh_build="host", **kw)
    rc = backend.lib().rt_session_create(C.byref(d), C.byref(p), C.byref(h))
    return rc, backend.lib().rt_last_error().decode()


def _one_triangle(s):
    mat = s.add_material(scene.matte((0.5, 0.5, 0.5)))
    s.add_instance(s.add_mesh([[0, 0, 1], [1, 0, 1], [0, 1, 1]], [[0, 1, 2]], st=[[0, 0], [1, 0], [0, 1]]), mat)
    return mat


def test_forward_input_rejected_on_host():
    s = scene.Scene(4, 4)
    mat = _one_triangle(s)
    s.add_mix(1, 0.0, 0.5)  # node 0 reads node 1
    s.add_checker((1, 1, 1), (0, 0, 0))
    s.bind_pattern(mat, "diffuseColor", 0)
    rc, msg = _create(s)
    assert rc == -1 and "lower index" in msg


def test_presence_binding_accepted_on_host():
    """Pattern-driven cutouts pass the host checks (the device decides them
    in shading and per shadow-ray blocker)."""
    s = scene.Scene(4, 4)
    mat = _one_triangle(s)
    s.bind_pattern(mat, "presence", s.add_checker((1, 1, 1), (0, 0, 0)))
    h = C.c_void_p()
    d = s.desc()
    p = abi.make_params(bvh_build="host")
    rc = backend.lib().rt_session_create(C.byref(d), C.byref(p), C.byref(h))
    msg = backend.lib().rt_last_error().decode()
    if rc == 0:
        backend.lib().rt_session_destroy(h)
    assert rc != -1, msg   # without a GPU the session stops at the device, not at the scene


def test_too_many_nodes_per_material_refused():
    s = scene.Scene(4, 4)
    mat = _one_triangle(s)
    first = s.add_checker((1, 1, 1), (0, 0, 0))
    for _ in range(15):
        s.add_fractal()
    last = s.add_mix(first, 0.0, 0.5)
    s.bind_pattern(mat, "diffuseColor", last)
    rc, msg = _create(s)
    assert rc == -1 and "16 consecutive" in msg


def test_binding_to_missing_node_refused():
    s = scene.Scene(4, 4)
    mat = _one_triangle(s)
    s.add_checker((1, 1, 1), (0, 0, 0))
    s.bind_pattern(mat, "diffuseColor", 5)
    rc, msg = _create(s)
    assert rc == -1 and "missing material, node or field" in msg
