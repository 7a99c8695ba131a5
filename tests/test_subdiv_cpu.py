"""Catmull-Clark subdivision of SubdivisionMesh cages (rtcuda/subdiv.py)
against the reference's own tests (src/geometry/subdiv.rs:360-472) and
the RIB SubdivisionMesh request with its tags."""
import numpy as np

from rtcuda.rib import load_rib_string
from rtcuda.subdiv import levels_for_shading_rate, tessellate

CUBE = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1],
                 [-1, 1, 1]], np.float64)
FACES = [[0, 1, 2, 3], [5, 4, 7, 6], [4, 0, 3, 7], [1, 5, 6, 2], [3, 2, 6, 7], [4, 5, 1, 0]]
RING = [(0, 1, 1e9), (1, 2, 1e9), (2, 3, 1e9), (3, 0, 1e9)]


def test_cube_rounds_toward_sphere():
    pos, idx, nrm = tessellate(CUBE, FACES, 3, interpolate_boundary=True)
    assert len(idx) > 500
    r = np.linalg.norm(pos.astype(np.float64), axis=1)
    assert r.max() < 1.5 and r.max() / r.min() < 1.35
    np.testing.assert_allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-6)
    # The normals follow the cage's winding (this cage is wound inward): all
    # on one side of the surface.
    side = np.einsum("ij,ij->i", nrm, pos)
    assert (side < 0).all() or (side > 0).all()


def test_infinite_crease_keeps_edge_sharp():
    pos, _, _ = tessellate(CUBE, FACES, 3, creases=RING, interpolate_boundary=True)
    plane = pos[np.abs(pos[:, 2] + 1.0) < 1e-4]
    assert len(plane) > 20
    assert np.abs(plane[:, :2]).max() > 0.9


def test_corner_tags_pin_vertices():
    pos, _, _ = tessellate(CUBE, FACES, 3, creases=RING, corners=[(v, 1e9) for v in range(4)],
                           interpolate_boundary=True)
    pinned = ((np.abs(np.abs(pos[:, 0]) - 1) < 1e-5) & (np.abs(np.abs(pos[:, 1]) - 1) < 1e-5) &
              (np.abs(pos[:, 2] + 1) < 1e-5))
    assert pinned.sum() >= 4


def test_hole_faces_removed():
    with_hole = len(tessellate(CUBE, FACES, 1, holes=[0], interpolate_boundary=True)[1])
    without = len(tessellate(CUBE, FACES, 1, interpolate_boundary=True)[1])
    assert with_hole < without


def test_semi_sharp_crease_between_smooth_and_sharp():
    # A sharpness-1 crease ring sits between the smooth and infinitely sharp results.
    def extent(creases):
        pos = tessellate(CUBE, FACES, 3, creases=creases, interpolate_boundary=True)[0]
        return np.abs(pos[np.abs(pos[:, 2] + 1.0) < 0.2][:, :2]).max()
    soft, semi, hard = extent([]), extent([(a, b, 1.0) for a, b, _ in RING]), extent(RING)
    assert soft < semi < hard


def test_rib_subdivision_mesh_tags_and_shading_rate():
    cage = ('"P" [-1 -1 -1  1 -1 -1  1 1 -1  -1 1 -1  -1 -1 1  1 -1 1  1 1 1  -1 1 1]')
    faces = "[4 4 4 4 4 4] [0 1 2 3  5 4 7 6  4 0 3 7  1 5 6 2  3 2 6 7  4 5 1 0]"
    s = load_rib_string(f'ShadingRate 4\nSubdivisionMesh "catmull-clark" {faces} '
                        f'["crease" "corner" "hole" "interpolateboundary"] [5 1 1 1 1 0 0 0] '
                        f'[0 1 2 3 0 0 5] [20 20] {cage}\n'
                        f'AttributeBegin ShadingRate 0.1\nSubdivisionMesh "loop" {faces} {cage}\nAttributeEnd')
    a, b = (s.meshes[m] for m in s.instance_array()["mesh"])
    ref = tessellate(CUBE, FACES, levels_for_shading_rate(4.0), creases=[(0, 1, 20), (1, 2, 20), (2, 3, 20),
                                                                         (3, 0, 20)],
                     corners=[(0, 20)], holes=[5], interpolate_boundary=True)
    np.testing.assert_array_equal(a[0], ref[0])
    np.testing.assert_array_equal(a[1], ref[1].astype(np.uint32))
    assert len(b[1]) == 6 * 4 ** 5 * 2  # level 5 at shading rate 0.1, no holes
    assert any("loop" in w for w in s.warnings)
