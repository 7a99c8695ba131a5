"""Participating media and subsurface scattering on the GPU against the f64
oracle (src/raytracer/pt/volume.rs, src/scene/medium.rs and the media and
subsurface branches of trace_full, src/raytracer/pt/mod.rs:480-892,
1244-1306), at the path tracer's image tolerance (tests/mc_parity.py): the
GPU image's relMSE against a high-spp oracle render within the Monte Carlo
interval of an independent oracle render's, and the mean of the oracle's
render of the same samples.

Each feature of the media Cornell box runs alone and then all together:
homogeneous fog with equiangular and collision NEE toward a point light,
an fBm cloud in a volume hull (delta and ratio tracking, hull crossings in
shadow rays), rough glass with an absorbing interior (nested media on
transmission), and the subsurface random walk."""
import numpy as np
import pytest

from mc_parity import compare, render_quad
from rtcuda import PtSession, RtError, abi, scenes

pytestmark = pytest.mark.gpu

ONLY = {
    "fog": dict(cloud=False, glass=False, sss=False),
    "cloud": dict(fog=False, glass=False, sss=False),
    "glass": dict(fog=False, cloud=False, sss=False),
    "sss": dict(fog=False, cloud=False, glass=False),
    "all": {},
}


@pytest.mark.parametrize("feature", list(ONLY))
def test_media_cornell_parity(feature):
    s = scenes.media_cornell(48, 48, **ONLY[feature])
    p = abi.make_params(max_depth=8)
    g, o, r, pr, st = render_quad(s, p, 32, 1024)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res
    assert st["extension_rays"] > 0


def test_absorbing_atmosphere_closed_form():
    """Camera rays through an absorbing slab atmosphere 2 units deep reach
    the background scaled by exp(-sigma_a * 2) per channel."""
    s = scenes.Scene(32, 32, fov=10.0)
    s.add_material(scenes.matte((0.5,) * 3))
    s.background = (1.0, 0.5, 0.25)
    s.add_medium(scenes.medium((0.2, 0.5, 1.0), (0.0, 0.0, 0.0), max_distance=2.0), atmosphere=True)
    with PtSession(s, abi.make_params(max_depth=4)) as g:
        g.render_samples(0, 256)
        img = g.image().reshape(-1, 3)
    want = np.array([1.0, 0.5, 0.25]) * np.exp(-np.array([0.2, 0.5, 1.0]) * 2.0)
    np.testing.assert_allclose(img.mean(0), want, rtol=0.01)


def test_media_render_same_seed_bitwise():
    """Media and walks keep renders reproducible: one thread adds both of a
    path's shadow contributions in a fixed order, and ratio tracking in
    shadow rays draws from a stream derived from the path's."""
    s = scenes.media_cornell(40, 40)
    p = abi.make_params(max_depth=8)
    imgs = []
    for _ in range(2):
        with PtSession(s, p) as g:
            g.render_samples(0, 8)
            imgs.append(g.image())
    assert np.array_equal(imgs[0], imgs[1])


def test_media_slab_size_invariance():
    """Whole sample passes per slab do not change the image."""
    s = scenes.media_cornell(32, 32)
    imgs = []
    for mp in (32 * 32, 8 * 32 * 32):
        with PtSession(s, abi.make_params(max_depth=8, max_paths=mp)) as g:
            g.render_samples(0, 8)
            imgs.append(g.image())
    assert np.array_equal(imgs[0], imgs[1])


def test_guided_media_rejected():
    s = scenes.media_cornell(16, 16, cloud=False, glass=False, sss=False)
    with pytest.raises(RtError) as e:
        PtSession(s, abi.make_params(max_depth=8, guided=True))
    assert e.value.code == -1 and "media" in str(e.value)
