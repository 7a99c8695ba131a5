"""Degenerate and ragged inputs on the GPU path: empty scenes, empty meshes,
zero-area triangles, one-pixel and one-row frames, zero-sample calls, the
maximum bounce count. The reference's tests cover the same corners on its
CPU path (empty BVH, degenerate triangles, sample-range edges)."""
import numpy as np
import pytest

import oracle
from rtcuda import PtSession, abi, scenes
from rtcuda.scene import Scene, matte

pytestmark = pytest.mark.gpu


def _box_scene(w=24, h=16):
    s = scenes.cornell_box(w, h)
    return s


def test_empty_scene_is_background():
    s = Scene(16, 8)
    s.background = (0.25, 0.5, 0.75)
    s.add_point_light((0, 1, 0), 5.0)
    with PtSession(s, abi.make_params(max_depth=8)) as g:
        g.render_samples(0, 4)
        img = g.image()
        st = g.stats()
    assert st["extension_rays"] == 16 * 8 * 4
    np.testing.assert_array_equal(img, np.broadcast_to(np.float32([0.25, 0.5, 0.75]), img.shape))


def test_empty_mesh_instance_changes_nothing():
    # An instance of a mesh with no triangles must not alter any hit.
    a = _box_scene()
    b = _box_scene()
    empty = b.add_mesh(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))
    b.add_instance(empty, 0)
    p = abi.make_params(max_depth=8)
    with PtSession(a, p) as ga, PtSession(b, p) as gb:
        ga.render_samples(3, 8)
        gb.render_samples(3, 8)
        assert np.array_equal(ga.sum_and_weight(), gb.sum_and_weight())


def test_zero_area_triangles_are_ignored():
    a = _box_scene()
    b = _box_scene()
    # Degenerate triangles (repeated vertices, collinear points) in front of the camera.
    pos = np.array([[0, 0, 0.5], [0, 0, 0.5], [0.3, 0.2, 0.5], [0, 0, 0.2], [0.1, 0.1, 0.2], [0.2, 0.2, 0.2]],
                   np.float32)
    idx = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    b.add_instance(b.add_mesh(pos, idx), b.add_material(matte((0.5, 0.5, 0.5))))
    p = abi.make_params(max_depth=8)
    with PtSession(a, p) as ga, PtSession(b, p) as gb:
        ga.render_samples(0, 8)
        gb.render_samples(0, 8)
        ia, ib = ga.image(), gb.image()
    assert np.isfinite(ib).all()
    assert np.array_equal(ia, ib)


@pytest.mark.parametrize("w,h", [(1, 1), (37, 1), (1, 29)])
def test_ragged_frames_match_oracle(w, h):
    s = _box_scene(w, h)
    p = abi.make_params(max_depth=8)
    spp = 512
    with PtSession(s, p) as g:
        g.render_samples(0, spp)
        img = g.image()
        assert g.sum_and_weight()[..., 3].min() == spp
    cpu = oracle.OracleScene(s).render(p, 0, spp)[0].reshape(h, w, 3) / spp
    mc, mg = cpu.mean((0, 1)), img.mean((0, 1))
    assert np.all(np.abs(mc - mg) <= 0.1 * mc + 0.02), (mc, mg)


def test_zero_sample_call_and_maximum_depth():
    s = _box_scene()
    with PtSession(s, abi.make_params(max_depth=255)) as g:
        g.render_samples(0, 0)
        assert g.sum_and_weight()[..., 3].max() == 0
        g.render_samples(0, 4)
        img = g.image()
        assert np.isfinite(img).all() and img.mean() > 0
