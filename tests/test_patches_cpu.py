"""PatchMesh / Patch dicing (rtcuda/patches.py) against the reference's
patch tests (src/geometry/patches.rs:338-380) and the RIB requests."""
import numpy as np

from rtcuda.patches import (BASES, basis_weights, bspline_basis, dice_segments, tessellate_bicubic,
                            tessellate_bilinear, tessellate_nurbs)
from rtcuda.rib import load_rib_string


def _grid(nu, nv, z=lambda x, y: 0.0 * x):
    x, y = np.meshgrid(np.linspace(0, 1, nu), np.linspace(0, 1, nv))
    return np.stack([x, y, z(x, y)], -1).reshape(-1)


def test_bases_partition_unity_and_bezier_endpoints():
    t = np.linspace(0, 1, 11)
    for name in ("bezier", "b-spline", "catmull-rom"):
        np.testing.assert_allclose(basis_weights(BASES[name][0], t).sum(1), 1.0, atol=1e-12)
    w = basis_weights(BASES["bezier"][0], np.array([0.0, 1.0]))
    np.testing.assert_allclose(w, [[1, 0, 0, 0], [0, 0, 0, 1]], atol=1e-12)


def test_bezier_patch_interpolates_corners():
    pts = _grid(4, 4, lambda x, y: np.sin(3 * x) * np.cos(2 * y))
    pos, idx, nrm, st = tessellate_bicubic(pts, 4, 4, False, False, BASES["bezier"], BASES["bezier"], 8)
    ctrl = pts.reshape(4, 4, 3)
    g = 9
    for (j, i), (cj, ci) in (((0, 0), (0, 0)), ((0, g - 1), (0, 3)), ((g - 1, 0), (3, 0)), ((g - 1, g - 1), (3, 3))):
        np.testing.assert_allclose(pos[j * g + i], ctrl[cj, ci], atol=1e-6)
    assert len(idx) == 8 * 8 * 2 and st.max() == 1.0


def test_bspline_mesh_multiple_patches_no_cracks():
    pts = _grid(7, 5, lambda x, y: x * y)
    pos, idx, _, _ = tessellate_bicubic(pts, 7, 5, False, False, BASES["b-spline"], BASES["b-spline"], 4)
    # 4 x 2 patches share one (4*4+1) x (2*4+1) vertex grid: no duplicates at seams.
    assert len(pos) == 17 * 9 and len(idx) == 16 * 8 * 2
    assert len(np.unique(pos.round(6), axis=0)) == len(pos)


def test_bilinear_and_wrap():
    pts = _grid(3, 2)
    pos, idx, _, st = tessellate_bilinear(pts, 3, 2, False, False, 4)
    assert len(pos) == 9 * 5 and len(idx) == 8 * 4 * 2
    np.testing.assert_allclose(pos[:, 2], 0.0)
    ring = np.stack([np.cos(a) for a in np.linspace(0, 2 * np.pi, 8, endpoint=False)])
    cyl = np.array([[np.cos(a), np.sin(a), z] for z in (0.0, 1.0)
                    for a in np.linspace(0, 2 * np.pi, 8, endpoint=False)]).reshape(-1)
    pos, idx, _, _ = tessellate_bilinear(cyl, 8, 2, True, False, 2)
    assert len(pos) == 16 * 3 and len(idx) == 16 * 2 * 2 and ring.shape == (8,)
    assert tessellate_bicubic(pts, 3, 2, False, False, BASES["bezier"], BASES["bezier"], 4) is None
    assert dice_segments(1.0) == 16 and dice_segments(100.0) == 2 and dice_segments(0.01) == 64


def test_rib_patch_requests():
    p16 = " ".join(f"{x:.3f}" for x in _grid(4, 4))
    s = load_rib_string(f'ShadingRate 4\nBasis "b-spline" 1 "catmull-rom" 1\n'
                        f'PatchMesh "bicubic" 4 "nonperiodic" 4 "nonperiodic" "P" [{p16}]\n'
                        f'Patch "bilinear" "P" [0 0 0  1 0 0  0 1 0  1 1 0]\n'
                        f'NuPatch 2 2 [0 0 1 1] 0 1 2 2 [0 0 1 1] 0 1 "P" [0 0 0 1 0 0 0 1 0 1 1 0]')
    inst = s.instance_array()
    assert len(inst) == 3  # the bicubic mesh, the bilinear patch, the NURBS sheet
    a = s.meshes[inst["mesh"][0]][0]
    ref = tessellate_bicubic(_grid(4, 4).round(3), 4, 4, False, False, BASES["b-spline"], BASES["catmull-rom"],
                             dice_segments(4.0))[0]
    np.testing.assert_allclose(a, ref, atol=1e-6)
    assert 0 in s.mesh_st and 1 in s.mesh_st and 2 in s.mesh_st
    sheet = s.meshes[inst["mesh"][2]][0]
    np.testing.assert_allclose(sheet[:, 2], 0.0) and np.testing.assert_allclose(sheet[0], [0, 0, 0], atol=1e-7)


def test_nurbs_flat_sheet():
    """patches.rs:380-417: an order-3 clamped sheet over a flat 4 x 3 net."""
    pts = [c for j in range(3) for i in range(4) for c in (i, j, 0.0)]
    pos, idx, _, _ = tessellate_nurbs(4, 3, [0, 0, 0, 0.5, 1, 1, 1], 0, 1, 3, 3, [0, 0, 0, 1, 1, 1], 0, 1, pts,
                                      False, 8, 8)
    assert np.abs(pos[:, 2]).max() < 1e-5
    assert pos[:, 0].min() >= -1e-5 and pos[:, 0].max() <= 3.0 + 1e-4
    assert abs(pos[0, 0]) < 1e-5 and abs(pos[0, 1]) < 1e-5
    # Clamped at both ends: the far corner too; bases sum to one inside.
    np.testing.assert_allclose(pos[-1], [3, 2, 0], atol=1e-5)
    for t in np.linspace(0, 1, 9):
        assert abs(bspline_basis([0, 0, 0, 0.5, 1, 1, 1], 4, 3, t).sum() - 1.0) < 1e-12


def test_bspline_basis_is_the_textbook_one():
    # Linear: N0 = 1 - t, N1 = t; quadratic Bezier-clamped: Bernstein polynomials.
    for t in (0.0, 0.3, 0.999):
        np.testing.assert_allclose(bspline_basis([0, 0, 1, 1], 2, 2, t), [1 - t, t], atol=1e-12)
        np.testing.assert_allclose(bspline_basis([0, 0, 0, 1, 1, 1], 3, 3, t),
                                   [(1 - t) ** 2, 2 * t * (1 - t), t * t], atol=1e-12)


def test_rational_nurbs_circle_arc():
    # A quarter circle as a rational quadratic (weights 1, sqrt(2)/2, 1), extruded in z.
    w = np.sqrt(0.5)
    row = [(1, 0, 1), (w * 1, w * 1, w), (0, 1, 1)]
    pts = [c for z in (0.0, 1.0) for (x, y, ww) in row for c in (x, y, z * ww, ww)]
    pos, _, _, _ = tessellate_nurbs(3, 3, [0, 0, 0, 1, 1, 1], 0, 1, 2, 2, [0, 0, 1, 1], 0, 1, pts, True, 8, 1)
    np.testing.assert_allclose(np.hypot(pos[:, 0], pos[:, 1]), 1.0, atol=1e-6)
