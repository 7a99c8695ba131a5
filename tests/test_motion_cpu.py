"""Motion blur on the host: the RIB route of the reference's MotionBegin
blocks (src/parser/scene_builder.rs:1637-1691, its test
motion_blocks_record_endpoints at :1951-1990), closed forms of moving
geometry rendered by the f64 oracle (Instance::transforms_at,
Mesh::vertex_at, Camera::apply_motion: src/geometry/mesh.rs:96-111,
295-304, src/scene/camera.rs:134-146), and the descriptor checks of the
C-ABI."""
import ctypes as C

import numpy as np

import oracle
from rtcuda import abi, backend, scene, scenes
from rtcuda.rib import load_rib_string


def test_rib_motion_blocks_record_endpoints():
    s = load_rib_string("""
        Format 64 64 1.0
        Shutter 0 1
        WorldBegin
            AttributeBegin
                MotionBegin [0 1]
                    Translate 0 0 5
                    Translate 2 0 5
                MotionEnd
                PointsPolygons [4] [0 1 2 3]
                    "P" [-1 -1 0  1 -1 0  1 1 0  -1 1 0]
            AttributeEnd
            AttributeBegin
                Translate 0 0 8
                MotionBegin [0 1]
                    PointsPolygons [4] [0 1 2 3] "P" [-1 -1 0  1 -1 0  1 1 0  -1 1 0]
                    PointsPolygons [4] [0 1 2 3] "P" [-1 -1 2  1 -1 2  1 1 2  -1 1 2]
                MotionEnd
            AttributeEnd
        WorldEnd
    """)
    assert s.has_motion
    assert s.n_instances == 2
    # Transform motion: the endpoint is shifted +2 in x.
    xf0 = s.instance_array()["xf"][0].reshape(3, 4)
    xf1 = s.instance_motion[0].reshape(3, 4)
    assert abs(xf1[0, 3] - xf0[0, 3] - 2.0) < 1e-9
    # Deformation motion: the second mesh carries positions at shutter close (+2 in z).
    p1 = s.mesh_motion[1]
    assert abs(p1[0, 2] - s.meshes[1][0][0, 2] - 2.0) < 1e-6
    assert 1 not in s.instance_motion


def test_rib_motion_applies_to_later_transforms():
    """motion_endpoint: transforms after the block compose onto both endpoints."""
    s = load_rib_string("""
        WorldBegin
            AttributeBegin
                MotionBegin [0 1]
                    Translate 0 0 0
                    Translate 1 0 0
                MotionEnd
                Translate 0 0 5
                Scale 2 2 2
                PointsPolygons [3] [0 1 2] "P" [0 0 0  1 0 0  0 1 0]
            AttributeEnd
            PointsPolygons [3] [0 1 2] "P" [0 0 0  1 0 0  0 1 0]
        WorldEnd
    """)
    xf0 = s.instance_array()["xf"][0].reshape(3, 4)
    xf1 = s.instance_motion[0].reshape(3, 4)
    np.testing.assert_allclose(xf0[:, :3], 2 * np.eye(3))
    np.testing.assert_allclose(xf1[:, :3], 2 * np.eye(3))
    np.testing.assert_allclose(xf1[:, 3] - xf0[:, 3], [1.0, 0.0, 0.0])
    assert 1 not in s.instance_motion   # after AttributeEnd the motion state is gone


def test_rib_camera_motion_is_the_inverse_delta():
    """A motion block over the pre-World transforms animates the camera:
    motion_inv = (t1 t0^-1)^-1 (scene_builder.rs:271-285)."""
    s = load_rib_string("""
        MotionBegin [0 1]
            Translate 0 0 3
            Translate 0.5 0 3
        MotionEnd
        WorldBegin
            PointsPolygons [3] [0 1 2] "P" [0 0 0  1 0 0  0 1 0]
        WorldEnd
    """)
    m = s.camera_motion_inv.reshape(3, 4)
    np.testing.assert_allclose(m[:, :3], np.eye(3), atol=1e-12)
    np.testing.assert_allclose(m[:, 3], [-0.5, 0.0, 0.0], atol=1e-12)
    assert not s.instance_motion   # the camera's block does not move world geometry


def test_rib_unsupported_motion_uses_first_sample():
    s = load_rib_string("""
        WorldBegin
            MotionBegin [0 1]
                Sphere 1 -1 1 360
                Sphere 2 -2 2 360
            MotionEnd
        WorldEnd
    """)
    assert any("MotionBegin" in w for w in s.warnings)
    assert len(s.quadrics) == 1 and s.quadrics[0][1][0] == 1.0


def _moving_quad(kind):
    """An emissive unit quad at z = 5 that crosses the view axis during the
    shutter (x from -1 to +1, or the rays move instead)."""
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
        s.camera_motion_inv = scene.affine(None, (-2.0, 0, 0))   # rays move by -2t in x
    return s


def test_moving_quad_covers_the_centre_half_the_shutter():
    """The quad (or the ray, under camera motion) moves 2 units across the
    centre ray over the shutter: the centre pixel sees it half the time."""
    spp = 4096
    for kind in ("transform", "deform", "camera"):
        img = oracle.OracleScene(_moving_quad(kind)).render(abi.make_params(max_depth=2), 0, spp)[0]
        c = img.reshape(9, 9, 3)[4, 4, 0] / spp
        assert abs(c - 0.5) < 4 * 0.5 / np.sqrt(spp), (kind, c)


def test_static_scene_draws_no_shutter_time():
    """Without motion no time is drawn: the image equals the same geometry
    described as a scene with every motion part switched off."""
    a = scenes.motion_cornell(16, 16, transform=False, deform=False, camera=False)
    assert not a.has_motion
    b = scenes.cornell_box(16, 16)
    p, i = scenes.quad((-0.2, -0.2, 0.4), (0.6, 0.0, 0.0), (0.0, 0.0, 0.5))
    b.add_instance(b.add_mesh(np.asarray(p, np.float32), i, normals=np.tile(np.float32([[0, 1, 0]]), (4, 1))),
                   b.add_material(scene.ggx_floor((0.8, 0.7, 0.3), 0.35)))
    prm = abi.make_params(max_depth=6)
    ia = oracle.OracleScene(a).render(prm, 0, 8)[0]
    ib = oracle.OracleScene(b).render(prm, 0, 8)[0]
    assert np.array_equal(ia, ib)


def test_motion_blur_changes_the_image():
    prm = abi.make_params(max_depth=6)
    moving = oracle.OracleScene(scenes.motion_cornell(16, 16)).render(prm, 0, 64)[0]
    still = oracle.OracleScene(scenes.motion_cornell(16, 16, transform=False, deform=False,
                                                     camera=False)).render(prm, 0, 64)[0]
    assert not np.array_equal(moving, still)


def _create(s, **kw):
    h = C.c_void_p()
    d = s.desc()
    p = abi.make_params(**kw)
    rc = backend.lib().rt_session_create(C.byref(d), C.byref(p), C.byref(h))
    return rc, backend.lib().rt_last_error().decode()


def test_bad_motion_descriptors_rejected_on_host():
    s = _moving_quad("transform")
    s.instance_motion[5] = s.instance_motion[0]
    rc, msg = _create(s)
    assert rc == -1 and "instance motion" in msg
    s = _moving_quad("deform")
    s.mesh_motion[0] = s.mesh_motion[0].copy()
    s.mesh_motion[0][0, 0] = np.inf
    s._desc = None
    rc, msg = _create(s)
    assert rc == -1 and "non-finite" in msg
    s = _moving_quad("camera")
    s.camera_motion_inv = np.full(12, np.nan)
    s._desc = None
    rc, msg = _create(s)
    assert rc == -1 and "camera motion" in msg
