"""Adaptive sampling (WfSession::set_adaptive): the stopping rule of the
reference's wavefront raygen, checked through properties that hold exactly,
plus statistical agreement with the f64 oracle's full render."""
import numpy as np
import pytest

import oracle
from rtcuda import PtSession, abi, scenes

pytestmark = pytest.mark.gpu


def test_tolerance_zero_changes_nothing():
    s = scenes.cornell_box(48, 48)
    p = abi.make_params(max_depth=8)
    with PtSession(s, p) as a, PtSession(s, p) as b:
        a.render_samples(0, 40)
        b.set_adaptive(0.0)
        b.render_samples(0, 40)
        assert b.average_spp() == 40.0
        assert np.array_equal(a.sum_and_weight(), b.sum_and_weight())


def test_huge_tolerance_stops_every_pixel_at_32():
    # From sample 32 on every pixel has n >= 16 and any interval is below a
    # huge tolerance: the render keeps exactly samples 0..31 of each pixel.
    s = scenes.cornell_box(48, 48)
    p = abi.make_params(max_depth=8)
    with PtSession(s, p) as a, PtSession(s, p) as b:
        a.set_adaptive(1e6)
        a.render_samples(0, 64)
        assert a.average_spp() == 32.0
        b.render_samples(0, 32)
        assert np.array_equal(a.sum_and_weight(), b.sum_and_weight())


def test_adaptive_spends_samples_where_noise_is():
    s = scenes.cornell_box(64, 64)
    p = abi.make_params(max_depth=8)
    spp = 256
    with PtSession(s, p) as g:
        g.set_adaptive(0.2)
        g.render_samples(0, spp)
        avg = g.average_spp()
        acc = g.sum_and_weight()
        img = g.image()
    n = acc[..., 3]
    # A pixel whose samples have a coefficient of variation c stops near
    # (1.96 c / 0.2)^2 samples: the noisy ones take many more than the flat.
    assert 32 <= n.min() and n.max() == spp
    assert 32 < avg < 0.8 * spp
    print(f"adaptive tol 0.2: {avg:.1f} spp on average of {spp}")
    # Pixels wholly inside the light see its radiance (17, 12, 4), luminance
    # 12.5, in every sample: zero variance, so they stop at the first check.
    lum = img @ np.array([0.2126, 0.7152, 0.0722])
    inside = np.abs(lum - 12.5) < 0.05
    assert inside.sum() > 4 and n[inside].max() == 32
    cpu = oracle.OracleScene(s).render(p, 0, 64)[0].reshape(64, 64, 3) / 64
    mc, mg = cpu.reshape(-1, 3).mean(0), img.reshape(-1, 3).mean(0)
    assert np.all(np.abs(mc - mg) / mc < 0.03), (mc, mg)
