"""Displacement at load time (src/geometry/displace.rs): the product's
numpy Perlin fBm (rtcuda/displace.py) against the oracle's C++ one (the
noise the fractal pattern reads), the reference's own noise test, and
the RIB Displace request on polygon meshes."""
import numpy as np

import oracle
from rtcuda import scene
from rtcuda.displace import displace_mesh, fbm, perlin, smooth_normals
from rtcuda.rib import load_rib_string


def _oracle_fbm(p, frequency, octaves, gain, lacunarity):
    s = scene.Scene(4, 4)
    node = s.add_fractal(frequency=frequency, octaves=octaves, gain=gain, lacunarity=lacunarity)
    ctx = np.hstack([np.zeros((len(p), 2)), p, np.zeros((len(p), 1))])
    return oracle.pattern_eval(s, node, ctx)[:, 0] * 2.0 - 1.0  # undo the pattern's 0.5 x + 0.5


def test_noise_matches_the_oracle():
    p = np.random.default_rng(5).uniform(-40.0, 40.0, (4000, 3))
    np.testing.assert_allclose(perlin(p), _oracle_fbm(p, 1.0, 1, 0.5, 2.0), atol=1e-12)
    f = fbm(p, frequency=0.7, octaves=5, gain=0.45, lacunarity=2.1)
    o = _oracle_fbm(p, 0.7, 5, 0.45, 2.1)
    inside = np.abs(f) < 0.999  # the pattern clamps to [0, 1]
    np.testing.assert_allclose(f[inside], o[inside], atol=1e-12)


def test_perlin_is_bounded_and_zero_at_lattice():
    """displace.rs:130-144."""
    lattice = np.array([[i, j, 0.0] for i in range(-3, 3) for j in range(-3, 3)])
    assert np.abs(perlin(lattice)).max() < 1e-12
    t = np.arange(1000) * 0.113
    mx = np.abs(perlin(np.stack([t, t * 0.7 + 0.3, t * 1.3 + 0.9], -1))).max()
    assert 0.05 < mx <= 1.3


def test_displace_mesh_moves_along_normals_and_rebuilds_them():
    x, y = np.meshgrid(np.linspace(-1, 1, 9), np.linspace(-1, 1, 9))
    P = np.stack([x.ravel(), y.ravel(), np.zeros(81)], -1).astype(np.float32)
    I = np.array([[r * 9 + c, r * 9 + c + 1, (r + 1) * 9 + c + 1] for r in range(8) for c in range(8)] +
                 [[r * 9 + c, (r + 1) * 9 + c + 1, (r + 1) * 9 + c] for r in range(8) for c in range(8)])
    Q, N = displace_mesh(P, I, None, amplitude=0.3, frequency=2.0)
    n0 = smooth_normals(P, I)
    expect = (P.astype(np.float64) + n0 * (fbm(P, 2.0) * 0.3)[:, None]).astype(np.float32)
    np.testing.assert_array_equal(Q, expect)
    assert np.abs(Q[:, 2]).max() > 0.01 and np.allclose(Q[:, :2], P[:, :2])
    np.testing.assert_allclose(np.linalg.norm(N, axis=1), 1.0, atol=1e-6)
    np.testing.assert_array_equal(N, smooth_normals(Q, I))


def test_rib_displace_request():
    quad = 'PointsPolygons [4] [0 1 2 3] "P" [-1 -1 0  1 -1 0  1 1 0  -1 1 0]\n'
    s = load_rib_string('AttributeBegin\nDisplace "noise" "amplitude" [0.5] "frequency" [3] "octaves" [2]\n' + quad +
                        'Sphere 1 -1 1 360\nAttributeEnd\n' + quad + 'Displace "bumps"\n')
    inst = s.instance_array()
    moved, plain = (s.meshes[m][0] for m in inst["mesh"])
    base = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], np.float32)
    n = smooth_normals(base, [[0, 1, 2], [0, 2, 3]])
    expect = (base + n * (fbm(base, 3.0, 2) * 0.5)[:, None]).astype(np.float32)
    np.testing.assert_allclose(moved, expect, atol=1e-7)
    np.testing.assert_array_equal(plain, base)  # AttributeEnd restored the state
    # the sphere stays an analytic quadric (the reference displaces meshes only)
    assert len(s.quadrics) == 1 and s.quadrics[0][1][:4] == [1.0, -1.0, 1.0, 360.0]
    assert any("bumps" in w for w in s.warnings)
