"""Camera projections on the host: the reference's camera unit test
ortho_rays_are_parallel (src/scene/camera.rs:203-211) through the oracle's
rays, the orthographic window from RIB Projection / ScreenWindow
(scene_builder.rs:495-534, 223-225), and an orthographic image's closed
form."""
import numpy as np

import oracle
from rtcuda import abi, scene, scenes
from rtcuda.rib import load_rib_string


def test_rib_orthographic_window():
    s = load_rib_string("""
        Format 64 32 1
        Projection "orthographic"
        ScreenWindow -3 3 -1.5 1.5
        WorldBegin
        WorldEnd
    """)
    assert s.projection == abi.PROJECTION_ORTHOGRAPHIC
    assert s.ortho_half == (3.0, 1.5)
    t = load_rib_string('Format 64 32 1\nProjection "orthographic"\nWorldBegin\nWorldEnd\n')
    assert t.ortho_half == (2.0, 1.0)   # Camera::new: (aspect, 1)


def test_ortho_rays_are_parallel_and_fill_the_window():
    """A 2 x 2 emissive square seen head-on through an orthographic window of
    half-extents (2, 2): it covers exactly the middle half of the frame in
    each axis (pixel centres), whatever its distance."""
    for z in (3.0, 30.0):
        s = scene.Scene(16, 16, fov=30.0)
        s.projection = abi.PROJECTION_ORTHOGRAPHIC
        s.ortho_half = (2.0, 2.0)
        em = s.add_material(scene.emitter((1.0, 1.0, 1.0)))
        p, i = scenes.quad((-1.0, -1.0, 0.0), (2, 0, 0), (0, 2, 0))
        s.add_instance(s.add_mesh(p, i), em, scene.affine(None, (0, 0, z)))
        s.filter, s.filter_width = abi.FILTER_BOX, 1e-3
        img = oracle.OracleScene(s).render(abi.make_params(max_depth=1), 0, 4)[0].reshape(16, 16, 3)[..., 0] / 4
        inside = np.zeros((16, 16), bool)
        inside[4:12, 4:12] = True
        assert np.array_equal(img > 0.5, inside), z
