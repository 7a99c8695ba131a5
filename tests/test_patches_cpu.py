"""PatchMesh / Patch dicing (rtcuda/patches.py) against the reference's
patch tests (src/geometry/patches.rs:338-380) and the RIB requests."""
import numpy as np

from rtcuda.patches import BASES, basis_weights, dice_segments, tessellate_bicubic, tessellate_bilinear
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
    assert len(inst) == 2
    a = s.meshes[inst["mesh"][0]][0]
    ref = tessellate_bicubic(_grid(4, 4).round(3), 4, 4, False, False, BASES["b-spline"], BASES["catmull-rom"],
                             dice_segments(4.0))[0]
    np.testing.assert_allclose(a, ref, atol=1e-6)
    assert 0 in s.mesh_st and 1 in s.mesh_st
    assert any("NuPatch" in w for w in s.warnings)
