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


def bspline_basis(knots, n_ctrl, order, t):
    """The n_ctrl B-spline basis values at t: the knot span holding t (the
    last one at the end of the range, as patches.rs:236-251 picks it), then
    the Cox-de Boor recursion up to degree order - 1 within that span. The
    in-place update runs upward (each N_i,p reads the old N_i,p-1 and
    N_i+1,p-1); the reference's runs downward and reads N_i+1,p instead,
    which for knots [0 0 1 1] gives N_0 = t (1 - t) rather than 1 - t."""
    k = [float(x) for x in knots]
    degree = order - 1
    basis = [0.0] * (n_ctrl + degree + 1)
    hi = min(n_ctrl, max(len(k) - order, 0))
    span = degree
    for i in range(degree, hi):
        if t < k[i + 1] or i == hi - 1:
            span = i
            break
        span = i + 1
    basis[span] = 1.0

    def knot(i):
        return k[i] if 0 <= i < len(k) else 0.0
    for p in range(1, degree + 1):
        for i in range(max(span - p, 0), span + 1):
            val = 0.0
            d1 = knot(i + p) - k[i]
            if d1 > 1e-12:
                val += basis[i] * (t - k[i]) / d1
            d2 = knot(i + p + 1) - knot(i + 1)
            if d2 > 1e-12:
                val += basis[i + 1] * (knot(i + p + 1) - t) / d2
            basis[i] = val
    return np.array(basis[:n_ctrl])


def tessellate_nurbs(nu, uorder, uknot, umin, umax, nv, vorder, vknot, vmin, vmax, points, rational, segs_u,
                     segs_v):
    """tessellate_nurbs (patches.rs:271-336): a (segs_u + 1) x (segs_v + 1)
    grid over [umin, umax] x [vmin, vmax]; rational points are homogeneous
    (w x, w y, w z, w)."""
    stride = 4 if rational else 3
    pts = np.asarray(points, dtype=np.float64)
    if len(pts) < nu * nv * stride:
        return None
    ctrl = pts[:nu * nv * stride].reshape(nv, nu, stride)
    us = umin + (umax - umin) * np.arange(segs_u + 1) / segs_u
    vs = vmin + (vmax - vmin) * np.arange(segs_v + 1) / segs_v
    bu = np.array([bspline_basis(uknot, nu, uorder, u) for u in us])  # (gu, nu)
    bv = np.array([bspline_basis(vknot, nv, vorder, v) for v in vs])  # (gv, nv)
    xyz = np.einsum("vj,ui,jic->vuc", bv, bu, ctrl[..., :3])
    if rational:
        w = np.einsum("vj,ui,ji->vu", bv, bu, ctrl[..., 3])
        xyz = np.where(np.abs(w)[..., None] > 1e-12, xyz / np.where(np.abs(w) > 1e-12, w, 1.0)[..., None], xyz)
    su = (np.arange(segs_u + 1) / segs_u).astype(np.float32)
    sv = (np.arange(segs_v + 1) / segs_v).astype(np.float32)
    return _mesh(xyz, segs_u + 1, segs_v + 1, False, False, su, sv)
