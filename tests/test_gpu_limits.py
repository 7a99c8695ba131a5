"""Bounded device loops running out, on the GPU, without a fault.

Every device loop that waits has a limit (rt_params.max_trav_steps and
wait_polls, rt_set_limits). A limit set tiny makes the loop run out: the
kernel records an error bit and ends its work, the call returns
RT_ERR_DEVICE with the loop named, and the CUDA context stays usable. The
reference's counterpart is its GPU watchdog retry
(src/raytracer/metal/renderer.rs:406-437).
"""
import numpy as np
import pytest

from rtcuda import PtSession, RtError, abi, scenes

pytestmark = pytest.mark.gpu


def test_traversal_step_limit_reports_and_session_recovers():
    s = scenes.cornell_box(48, 48)
    p = abi.make_params(max_depth=8)
    with PtSession(s, p) as fresh:
        fresh.render_samples(0, 4)
        want = fresh.image()
    with PtSession(s, p) as g:
        g.set_limits(max_trav_steps=2)
        with pytest.raises(RtError) as e:
            g.render_samples(0, 4)
        assert e.value.code == -4 and "step limit" in str(e.value)
        # The same session, limits back to their defaults: reset, render again.
        g.set_limits()
        g.reset()
        g.render_samples(0, 4)
        assert np.array_equal(g.image(), want)
        # and the ray-batch path reports the same way
        rays = scenes.triangle_cloud_rays(4096, seed=3)
        g.set_limits(max_trav_steps=1)
        with pytest.raises(RtError) as e:
            g.intersect(rays)
        assert e.value.code == -4
        g.set_limits()
        g.intersect(rays)


def test_tensor_core_wait_limit_reports_and_context_survives():
    """One poll per pipeline wait in the learned proposal's tcgen05 kernels:
    the waits run out (the MMAs they issued are drained before the kernel
    frees its TMEM), the render returns RT_ERR_DEVICE, and a new guided
    session on the same device then trains and renders normally."""
    s = scenes.two_rooms(64, 36)
    with PtSession(s, abi.make_params(max_depth=16, guided=True, wait_polls=1)) as g:
        with pytest.raises(RtError) as e:
            g.render_samples(0, 2)
        assert e.value.code == -4 and "tensor-core" in str(e.value)
    with PtSession(s, abi.make_params(max_depth=16, guided=True)) as g:
        g.render_samples(0, 4)
        img = g.image()
        assert g.stats()["guide_steps"] > 0
    assert np.isfinite(img).all() and img.mean() > 0
