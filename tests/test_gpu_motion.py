"""Motion blur on the GPU against the f64 oracle: transform motion
(Instance::transforms_at, src/geometry/mesh.rs:295-304), deformation
(Mesh::vertex_at and the geometric normal at the shutter time,
mesh.rs:96-111, 200-220) and camera motion (Camera::apply_motion,
src/scene/camera.rs:134-146), with the shutter time drawn after the filter
and lens samples (src/raytracer/pt/mod.rs:339-356). Closed forms of a quad
crossing the view axis, then images at the path tracer's tolerance
(tests/mc_parity.py): each kind of motion alone and all together, the RIB
route of MotionBegin blocks, and same-seed reproducibility."""
import numpy as np
import pytest

from mc_parity import compare, render_quad
from rtcuda import PtSession, abi, scene, scenes

pytestmark = pytest.mark.gpu


def _moving_quad(kind):
    s = scene.Scene(9, 9, fov=20.0)
    em = s.add_material(scene.emitter((1.0, 1.0, 1.0)))
    p, i = scenes.quad((-0.5, -0.5, 0.0), (1, 0, 0), (0, 1, 0))
    p = np.asarray(p, np.float32)
    if kind == "transform":
        s.add_instance(s.add_mesh(p, i), em, scene.affine(None, (-1.0, 0, 5)), scene.affine(None, (1.0, 0, 5)))
    elif kind == "deform":
        m = s.add_mesh(p + np.float32([-1, 0, 0]), i, positions1=p + np.float32([1, 0, 0]))
        s.add_instance(m, em, scene.affine(None, (0, 0, 5)))
    else:
        s.add_instance(s.add_mesh(p, i), em, scene.affine(None, (-1.0, 0, 5)))
        s.camera_motion_inv = scene.affine(None, (-2.0, 0, 0))
    return s


@pytest.mark.parametrize("kind", ["transform", "deform", "camera"])
def test_moving_quad_covers_the_centre_half_the_shutter(kind):
    spp = 16384
    with PtSession(_moving_quad(kind), abi.make_params(max_depth=2)) as g:
        g.render_samples(0, spp)
        img = g.image().reshape(9, 9, 3)
    assert abs(img[4, 4, 0] - 0.5) < 4 * 0.5 / np.sqrt(spp), img[4, 4, 0]
    # The blur is symmetric about the centre column.
    np.testing.assert_allclose(img[4, :, 0], img[4, ::-1, 0], atol=6 * 0.5 / np.sqrt(spp))


PARTS = {
    "transform": dict(deform=False, camera=False),
    "deform": dict(transform=False, camera=False),
    "camera": dict(transform=False, deform=False),
    "all": {},
}


@pytest.mark.parametrize("part", list(PARTS))
def test_motion_cornell_parity(part):
    s = scenes.motion_cornell(48, 48, **PARTS[part])
    g, o, r, pr, st = render_quad(s, abi.make_params(max_depth=8), 32, 1024)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res


def test_rib_motion_parity():
    from rtcuda.rib import load_rib_string
    s = load_rib_string("""
Format 48 32 1
Projection "perspective" "fov" [40]
MotionBegin [0 1]
    Translate 0 0 0
    Translate 0.1 0 0
MotionEnd
WorldBegin
  Light "PxrDomeLight" "sky" "intensity" [0.6]
  AttributeBegin
    Bxdf "PxrSurface" "a" "diffuseColor" [0.8 0.3 0.2]
    MotionBegin [0 1]
      Translate -0.6 0 4
      Translate 0.2 0.3 4
    MotionEnd
    PointsPolygons [4] [0 1 2 3] "P" [-0.4 -0.4 0  0.4 -0.4 0  0.4 0.4 0  -0.4 0.4 0]
  AttributeEnd
  AttributeBegin
    Bxdf "PxrSurface" "b" "diffuseColor" [0.2 0.5 0.8]
    Translate 0.6 0 4.5
    MotionBegin [0 1]
      PointsPolygons [4] [0 1 2 3] "P" [-0.3 -0.3 0  0.3 -0.3 0  0.3 0.3 0  -0.3 0.3 0]
      PointsPolygons [4] [0 1 2 3] "P" [-0.3 -0.3 -0.5  0.3 -0.3 0  0.3 0.6 0  -0.3 0.3 0.4]
    MotionEnd
  AttributeEnd
WorldEnd
""")
    assert s.has_motion and s.instance_motion and s.mesh_motion and s.camera_motion_inv is not None
    g, o, r, pr, _ = render_quad(s, abi.make_params(max_depth=6), 32, 1024)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res


def test_motion_same_seed_bitwise():
    s = scenes.motion_cornell(40, 40)
    imgs = []
    for _ in range(2):
        with PtSession(s, abi.make_params(max_depth=8)) as g:
            g.render_samples(0, 8)
            imgs.append(g.image())
    assert np.array_equal(imgs[0], imgs[1])


def test_motion_slab_size_invariance():
    s = scenes.motion_cornell(32, 32)
    imgs = []
    for mp in (32 * 32, 8 * 32 * 32):
        with PtSession(s, abi.make_params(max_depth=8, max_paths=mp)) as g:
            g.render_samples(0, 8)
            imgs.append(g.image())
    assert np.array_equal(imgs[0], imgs[1])


def test_motion_with_aovs_parity():
    """The first-surface AOV path (cutouts and skips in shading waves) with
    motion: the beauty image still matches the oracle."""
    s = scenes.motion_cornell(40, 40)
    g, o, r, pr, _ = render_quad(s, abi.make_params(max_depth=8, aovs=1), 32, 1024)
    res = compare(g, o, r, paired=pr)
    assert res["ok"], res


def test_motion_with_media_and_guiding_run():
    """Motion in a scene with fog and a subsurface walk (medium-aware shadow
    walks and walks carry the path's time), and in a guided render: finite
    images, reproducible."""
    s = scenes.media_cornell(32, 32, cloud=False, glass=False)
    s.camera_motion_inv = scene.affine(None, (-0.1, 0.0, 0.0))
    s.instance_motion[3] = s.instance_array()["xf"][3] + np.array([0, 0, 0, 0.2, 0, 0, 0, 0, 0, 0, 0, 0])
    imgs = []
    for _ in range(2):
        with PtSession(s, abi.make_params(max_depth=8)) as g:
            g.render_samples(0, 16)
            imgs.append(g.image())
    assert np.isfinite(imgs[0]).all() and imgs[0].mean() > 0
    assert np.array_equal(imgs[0], imgs[1])
    m = scenes.motion_cornell(32, 32)
    with PtSession(m, abi.make_params(max_depth=8, guided=True)) as g:
        g.render_samples(0, 8)
        img = g.image()
    assert np.isfinite(img).all() and img.mean() > 0
