"""Bilinear and bicubic PatchMesh / Patch dicing, as the reference's scene
builder tessellates them (src/geometry/patches.rs): RenderMan basis
matrices with their steps, wrapped (periodic) or open control grids, a
shared sample grid per mesh (crack-free across patches) with st running
over the whole mesh, area-weighted smooth normals."""
import numpy as np

from .displace import smooth_normals

# The RenderMan Interface basis matrices (rows multiply (t^3, t^2, t, 1))
# and their default steps.
_SIXTH = 1.0 / 6.0
BASES = {
    "bezier": (np.array([[-1, 3, -3, 1], [3, -6, 3, 0], [-3, 3, 0, 0], [1, 0, 0, 0]], np.float64), 3),
    "b-spline": (np.array([[-1, 3, -3, 1], [3, -6, 3, 0], [-3, 0, 3, 0], [1, 4, 1, 0]], np.float64) * _SIXTH, 1),
    "catmull-rom": (np.array([[-1, 3, -3, 1], [2, -5, 4, -1], [-1, 0, 1, 0], [0, 2, 0, 0]], np.float64) * 0.5, 1),
    "hermite": (np.array([[2, 1, -2, 1], [-3, -2, 3, -1], [0, 1, 0, 0], [1, 0, 0, 0]], np.float64), 2),
    "power": (np.eye(4), 4),
}
BASES["bspline"] = BASES["b-spline"]
BASES["catmullrom"] = BASES["catmull-rom"]


def basis_weights(m, t):
    """(t^3, t^2, t, 1) @ m for an array of t: (n, 4)."""
    t = np.asarray(t, dtype=np.float64)
    return np.stack([t ** 3, t ** 2, t, np.ones_like(t)], -1) @ m


def _grid_axes(n_patch, segs, wrap):
    """Per sample along one axis: patch index, local parameter, st."""
    g = n_patch * segs + (0 if wrap else 1)
    k = np.arange(g)
    patch = np.minimum(k // segs, n_patch - 1)
    local = k / segs - patch
    return patch, local, (k / (n_patch * segs)).astype(np.float32), g


def _triangulate(gu, gv, wrap_u, wrap_v):
    cu = np.arange(gu if wrap_u else gu - 1)
    cv = np.arange(gv if wrap_v else gv - 1)
    CV, CU = np.meshgrid(cv, cu, indexing="ij")
    a = CV * gu + CU
    b = CV * gu + (CU + 1) % gu
    c = ((CV + 1) % gv) * gu + (CU + 1) % gu
    d = ((CV + 1) % gv) * gu + CU
    return np.stack([a, b, c, a, c, d], -1).reshape(-1, 3)


def _mesh(P, gu, gv, wrap_u, wrap_v, su, sv):
    pos = P.astype(np.float32).reshape(-1, 3)
    idx = _triangulate(gu, gv, wrap_u, wrap_v)
    st = np.stack(np.broadcast_arrays(su[None, :], sv[:, None]), -1).reshape(-1, 2)
    return pos, idx, smooth_normals(pos, idx), st


def tessellate_bicubic(points, nu, nv, u_wrap, v_wrap, basis_u, basis_v, segs):
    """tessellate_bicubic (patches.rs:92-160); basis_* = (matrix, step).
    None for an invalid control grid."""
    pts = np.asarray(points, dtype=np.float64)
    if len(pts) < nu * nv * 3 or (nu < 4 and not u_wrap) or (nv < 4 and not v_wrap):
        return None
    (mu, ustep), (mv, vstep) = basis_u, basis_v
    npu = nu // ustep if u_wrap else (nu - 4) // ustep + 1
    npv = nv // vstep if v_wrap else (nv - 4) // vstep + 1
    if npu <= 0 or npv <= 0:
        return None
    ctrl = pts[:nu * nv * 3].reshape(nv, nu, 3)
    pu, lu, su, gu = _grid_axes(npu, segs, u_wrap)
    pv, lv, sv, gv = _grid_axes(npv, segs, v_wrap)
    wu, wv = basis_weights(mu, lu), basis_weights(mv, lv)  # (gu, 4), (gv, 4)
    P = np.zeros((gv, gu, 3))
    for jj in range(4):
        rows = (pv * vstep + jj) % nv
        for ii in range(4):
            cols = (pu * ustep + ii) % nu
            P += ctrl[rows][:, cols] * (wv[:, jj][:, None] * wu[:, ii][None, :])[..., None]
    return _mesh(P, gu, gv, u_wrap, v_wrap, su, sv)


def tessellate_bilinear(points, nu, nv, u_wrap, v_wrap, segs):
    """tessellate_bilinear (patches.rs:162-212)."""
    pts = np.asarray(points, dtype=np.float64)
    if len(pts) < nu * nv * 3 or nu < 2 or nv < 2:
        return None
    ctrl = pts[:nu * nv * 3].reshape(nv, nu, 3)
    pu, lu, su, gu = _grid_axes(nu if u_wrap else nu - 1, segs, u_wrap)
    pv, lv, sv, gv = _grid_axes(nv if v_wrap else nv - 1, segs, v_wrap)
    c00 = ctrl[pv % nv][:, pu % nu]
    c10 = ctrl[pv % nv][:, (pu + 1) % nu]
    c01 = ctrl[(pv + 1) % nv][:, pu % nu]
    c11 = ctrl[(pv + 1) % nv][:, (pu + 1) % nu]
    u, v = lu[None, :, None], lv[:, None, None]
    P = (c00 * (1.0 - u) + c10 * u) * (1.0 - v) + (c01 * (1.0 - u) + c11 * u) * v
    return _mesh(P, gu, gv, u_wrap, v_wrap, su, sv)


def dice_segments(shading_rate):
    """dice_segments (scene_builder.rs:1173-1175)."""
    return int(min(max(16.0 / max(shading_rate, 0.05), 2.0), 64.0))
