"""Camera rays on the GPU against the f64 oracle (src/scene/camera.rs:
36-61 pixel filters, 150-179 thin lens): triangle and Gaussian filters
spread samples beyond the pixel, the thin lens defocuses what is off the
focal plane. The GPU image agrees with the oracle's image of the same
camera in mean and profile, and is closer to it than to the oracle's
box-filtered pinhole image (so the camera model is really applied)."""
import numpy as np
import pytest

import oracle
from rtcuda import PtSession, abi, scenes

pytestmark = pytest.mark.gpu

SPP = 1024


@pytest.fixture(scope="module")
def pinhole_box():
    s = scenes.cornell_box(40, 40)
    return oracle.OracleScene(s).render(abi.make_params(max_depth=6), 0, SPP)[0].reshape(40, 40, 3) / SPP


@pytest.mark.parametrize("filt,width,lens", [(abi.FILTER_TRIANGLE, 2.0, 0.0), (abi.FILTER_GAUSSIAN, 1.5, 0.0),
                                             (abi.FILTER_BOX, 1.0, 0.12)],
                         ids=["triangle", "gaussian", "thin_lens"])
def test_camera_models_match_oracle(filt, width, lens, pinhole_box):
    s = scenes.cornell_box(40, 40)
    s.filter, s.filter_width = filt, width
    if lens:
        s.lens_radius, s.focal_distance = lens, 2.0
    p = abi.make_params(max_depth=6)
    with PtSession(s, p) as g:
        g.render_samples(0, SPP)
        img = g.image()
    cpu = oracle.OracleScene(s).render(p, 0, SPP)[0].reshape(40, 40, 3) / SPP
    np.testing.assert_allclose(img.mean((0, 1)), cpu.mean((0, 1)), rtol=0.02)
    for axis in (0, 1):
        a, b = img.mean(axis).mean(-1), cpu.mean(axis).mean(-1)
        assert np.all(np.abs(a - b) <= 0.08 * b + 0.015), (axis, np.abs(a - b).max())
    same, other = np.abs(img - cpu).mean(), np.abs(img - pinhole_box).mean()
    assert same < 0.8 * other, (same, other)


def test_orthographic_camera_matches_oracle():
    """Orthographic rays (camera.rs:154-159) from a window of half-extents
    (1.2, 1.2) over the Cornell box: image parity with the oracle
    (tests/mc_parity.py)."""
    from mc_parity import compare, render_quad
    s = scenes.cornell_box(40, 40)
    s.projection = abi.PROJECTION_ORTHOGRAPHIC
    s.ortho_half = (1.2, 1.2)
    g, o, r, pr, _ = render_quad(s, abi.make_params(max_depth=6), 32, 1024)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res
