"""GeneralPolygon ear clipping with holes (rtcuda/earclip.py) against the
reference's tests (src/geometry/earclip.rs:195-250) and the RIB request."""
import numpy as np

from rtcuda.earclip import triangulate_with_holes
from rtcuda.rib import load_rib_string


def _area(P, I):
    return 0.5 * np.linalg.norm(np.cross(P[I[:, 1]] - P[I[:, 0]], P[I[:, 2]] - P[I[:, 0]]), axis=1).sum()


def test_concave_polygon():
    outline = [[0, 0, 0], [2, 0, 0], [2, 1, 0], [1, 1, 0], [1, 2, 0], [0, 2, 0]]
    P, I = triangulate_with_holes([outline])
    assert len(I) == 4 and abs(_area(P, I) - 3.0) < 1e-9


def test_square_with_hole():
    outer = [[0, 0, 0], [4, 0, 0], [4, 4, 0], [0, 4, 0]]
    hole = [[1, 1, 0], [3, 1, 0], [3, 3, 0], [1, 3, 0]]
    P, I = triangulate_with_holes([outer, hole])
    assert abs(_area(P, I) - 12.0) < 1e-6


def test_tilted_polygon_and_rib():
    # An L-shape in the x = 1 plane (Newell axis x) with a square hole, via RIB.
    s = load_rib_string('GeneralPolygon [6 4] "P" [1 0 0  1 4 0  1 4 2  1 2 2  1 2 4  1 0 4  '
                        '1 0.5 0.5  1 1.5 0.5  1 1.5 1.5  1 0.5 1.5]')
    P, I, N = s.meshes[0]
    assert abs(_area(P.astype(np.float64), I.astype(np.int64)) - (12.0 - 1.0)) < 1e-5
    np.testing.assert_allclose(np.abs(N[:, 0]), 1.0, atol=1e-6)
