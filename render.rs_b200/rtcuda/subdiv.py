"""Uniform Catmull-Clark subdivision of SubdivisionMesh cages, as the
reference's scene builder dices them (src/geometry/subdiv.rs): face points,
edge points (midpoints on boundaries and sharp creases, blended for
semi-sharp ones), vertex points by the smooth rule (F + 2M + (n-3)P)/n,
the crease rule (6P + A + B)/8 along two sharp (or pinned boundary) edges,
pinned at corners and crease junctions; sharpness decays by one per level
(>= 10 counts as infinite); hole faces drop out; the result is
fan-triangulated with area-weighted smooth normals."""
import numpy as np

from .displace import smooth_normals

INFINITE = 1e9


def _key(a, b):
    return (a, b) if a < b else (b, a)


def subdivide_once(P, faces, creases, corners, holes, interpolate_boundary):
    """One round (subdiv.rs:87-286). P: list of f64 triples; faces: vertex
    rings; creases: {(a, b): sharpness}; corners: {v: sharpness}."""
    edge_faces, vertex_edges, vertex_faces = {}, {}, {}
    for fi, f in enumerate(faces):
        for i, a in enumerate(f):
            b = f[(i + 1) % len(f)]
            k = _key(a, b)
            edge_faces.setdefault(k, []).append(fi)
            for v in (a, b):
                lst = vertex_edges.setdefault(v, [])
                if k not in lst:
                    lst.append(k)
            vf = vertex_faces.setdefault(a, [])
            if fi not in vf:
                vf.append(fi)
    Pn = np.asarray(P, dtype=np.float64)
    out = [Pn[f].sum(0) / len(f) for f in faces]  # face points
    face_pt = list(range(len(faces)))
    edge_pt = {}
    for k, fs in edge_faces.items():
        a, b = Pn[k[0]], Pn[k[1]]
        mid = (a + b) * 0.5
        sharp = creases.get(k, 0.0)
        if len(fs) < 2 or sharp >= 1.0:
            pt = mid
        else:
            fp = sum(out[face_pt[f]] for f in fs)
            smooth = (a + b + fp) / (2.0 + len(fs))
            pt = smooth + (mid - smooth) * min(sharp, 1.0) if sharp > 0.0 else smooth
        out.append(pt)
        edge_pt[k] = len(out) - 1
    vert_pt = []
    for v in range(len(Pn)):
        p = Pn[v]
        edges = vertex_edges.get(v, [])
        vfaces = vertex_faces.get(v, [])
        boundary = [e for e in edges if len(edge_faces.get(e, ())) < 2]
        sharp = [(e, creases[e]) for e in edges if creases.get(e, 0.0) > 0.0]
        cs = corners.get(v, 0.0)

        def smooth_point():
            n = float(max(len(edges), 1))
            favg = sum((out[face_pt[f]] for f in vfaces), np.zeros(3)) / max(len(vfaces), 1)
            mavg = sum(((Pn[e[0]] + Pn[e[1]]) * 0.5 for e in edges), np.zeros(3)) / n
            return (favg + mavg * 2.0 + p * (n - 3.0)) / n

        def crease_point(pair):
            other = [e[1] if e[0] == v else e[0] for e in pair]
            return (p * 6.0 + Pn[other[0]] + Pn[other[1]]) / 8.0

        if cs >= 1.0:
            pt = p
        elif interpolate_boundary and len(boundary) >= 2:
            pt = crease_point(boundary[:2])
        elif len(sharp) >= 3:
            pt = p
        elif len(sharp) == 2:
            avg = (sharp[0][1] + sharp[1][1]) * 0.5
            cp = crease_point([sharp[0][0], sharp[1][0]])
            pt = cp if avg >= 1.0 else smooth_point() + (cp - smooth_point()) * avg
        else:
            sp = smooth_point()
            pt = sp + (p - sp) * min(cs, 1.0) if cs > 0.0 else sp
        out.append(pt)
        vert_pt.append(len(out) - 1)
    new_faces = []
    for fi, f in enumerate(faces):
        if fi in holes:
            continue
        n = len(f)
        for i in range(n):
            prev, cur, nxt = f[(i + n - 1) % n], f[i], f[(i + 1) % n]
            new_faces.append([vert_pt[cur], edge_pt[_key(cur, nxt)], face_pt[fi], edge_pt[_key(prev, cur)]])
    new_creases = {}
    for (a, b), s in creases.items():
        ns = s - 1.0
        if ns > 0.0 and (a, b) in edge_pt:
            new_creases[_key(vert_pt[a], edge_pt[(a, b)])] = ns
            new_creases[_key(vert_pt[b], edge_pt[(a, b)])] = ns
    new_corners = {}
    for v, s in corners.items():
        if s - 1.0 > 0.0 or s >= INFINITE:
            new_corners[vert_pt[v]] = s if s >= INFINITE else s - 1.0
    return out, new_faces, new_creases, new_corners


def tessellate(P, faces, levels, creases=(), corners=(), holes=(), interpolate_boundary=False):
    """SubdivCage::tessellate (subdiv.rs:288-326): (positions f32, triangle
    indices, smooth normals). creases: (a, b, sharpness) triples; corners:
    (vertex, sharpness) pairs; sharpness >= 10 is infinite."""
    cr = {}
    for a, b, s in creases:
        cr[_key(int(a), int(b))] = INFINITE if s >= 10.0 else max(float(s), 0.0)
    co = {int(v): (INFINITE if s >= 10.0 else max(float(s), 0.0)) for v, s in corners}
    pts = [np.asarray(p, dtype=np.float64) for p in np.asarray(P, dtype=np.float64).reshape(-1, 3)]
    fcs = [[int(v) for v in f] for f in faces]
    hl = set(int(h) for h in holes)
    for _ in range(levels):
        pts, fcs, cr, co = subdivide_once(pts, fcs, cr, co, hl, interpolate_boundary)
        hl = set()
    pos = np.asarray(pts, dtype=np.float64).astype(np.float32).reshape(-1, 3)
    tris = [(f[0], f[i], f[i + 1]) for f in fcs for i in range(1, len(f) - 1)]
    idx = np.asarray(tris, dtype=np.int64).reshape(-1, 3)
    return pos, idx, smooth_normals(pos, idx) if len(idx) else np.zeros_like(pos)


def levels_for_shading_rate(rate):
    """subdiv_levels (scene_builder.rs:1178-1191)."""
    return 5 if rate <= 0.15 else 4 if rate <= 0.35 else 3 if rate <= 1.5 else 2 if rate <= 6.0 else 1
