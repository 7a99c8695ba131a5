"""The Monte Carlo parity check (tests/mc_parity.py) on oracle renders alone,
and the oracle's shadow transmittance, without a GPU.

Two independent oracle renders at the same spp pass the check; a planted
mistake in one of them (a 1% scale against its paired render, or fewer
samples per pixel, i.e. more variance) fails it."""
import numpy as np

import oracle
from mc_parity import compare
from rtcuda import abi, scene, scenes


def _renders():
    s = scenes.cornell_box(48, 48)
    o_s = oracle.OracleScene(s)
    p = abi.make_params(max_depth=8)
    a = o_s.render(p, 1 << 20, (1 << 20) + 16)[0] / 16
    b = o_s.render(p, 1 << 22, (1 << 22) + 16)[0] / 16
    few = o_s.render(p, 1 << 21, (1 << 21) + 4)[0] / 4
    ref = o_s.render(p, 1 << 23, (1 << 23) + 256)[0] / 256
    return a, b, few, ref


def test_same_distribution_passes_and_planted_mistakes_fail():
    a, b, few, ref = _renders()
    assert compare(a, b, ref)["ok"]
    assert compare(a, b, ref, paired=a)["ok"]
    # a 1% scale: far inside the image noise, caught by the paired check
    biased = compare(a * 1.01, b, ref, paired=a)
    assert not biased["ok"], biased
    noisy = compare(few, b, ref)
    assert not noisy["ok"] and noisy["relmse_diff"] > 0, noisy


def test_oracle_transmittance_multiplies_cutouts():
    s = scene.Scene(4, 4)
    half = s.add_material(scene.matte((0.5,) * 3, presence=0.5))
    quarter = s.add_material(scene.matte((0.5,) * 3, presence=0.75))
    solid = s.add_material(scene.matte((0.5,) * 3))
    quad = s.add_mesh([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], [[0, 1, 2], [0, 2, 3]])
    s.add_instance(quad, half, scene.affine(np.eye(3), (0, 0, 1)))
    s.add_instance(quad, quarter, scene.affine(np.eye(3), (0, 0, 2)))
    s.add_instance(quad, solid, scene.affine(np.eye(3), (0, 0, 3)))
    planes = np.zeros((2, 3, 4), np.float32)
    planes[1, :, :3] = (0, 0, 1)
    planes[1, :, 3] = (1.5, 2.5, 3.5)       # crosses 1, 2, then 3 quads
    t = oracle.OracleScene(s).transmittance(planes)[:, 0]
    np.testing.assert_allclose(t, [0.5, 0.5 * 0.25, 0.0], atol=1e-12)
