"""GeneralPolygon triangulation with holes, as the reference's scene
builder does it (src/geometry/earclip.rs): the loops are projected onto the
dominant plane of the outline's Newell normal, the outline is made
counter-clockwise and each hole clockwise, each hole is bridged into the
outline from its largest-x vertex to the nearest outline vertex whose
bridge crosses no edge, then convex ears holding no other vertex are
clipped (any remainder is fanned)."""
import numpy as np


def _cross(o, a, b):
    return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])


def _area(p):
    return 0.5 * sum(p[i][0] * p[(i + 1) % len(p)][1] - p[(i + 1) % len(p)][0] * p[i][1] for i in range(len(p)))


def _inside(p, a, b, c):
    d = (_cross(p, a, b), _cross(p, b, c), _cross(p, c, a))
    return not (any(x < 0.0 for x in d) and any(x > 0.0 for x in d))


def _crossing(a, b, c, d):
    d1, d2, d3, d4 = _cross(c, d, a), _cross(c, d, b), _cross(a, b, c), _cross(a, b, d)
    return ((d1 > 0.0 > d2) or (d1 < 0.0 < d2)) and ((d3 > 0.0 > d4) or (d3 < 0.0 < d4))


def triangulate_with_holes(loops):
    """(positions (n, 3) f64, triangle indices (m, 3)) or None."""
    outline = [tuple(map(float, p)) for p in loops[0]]
    n = np.zeros(3)
    for i in range(len(outline)):
        a, b = outline[i], outline[(i + 1) % len(outline)]
        n += [(a[1] - b[1]) * (a[2] + b[2]), (a[2] - b[2]) * (a[0] + b[0]), (a[0] - b[0]) * (a[1] + b[1])]
    an = np.abs(n)
    axis = 0 if an[0] >= an[1] and an[0] >= an[2] else (1 if an[1] >= an[2] else 2)
    keep = {0: (1, 2), 1: (2, 0), 2: (0, 1)}[axis]

    def project(pts):
        return [(p[keep[0]], p[keep[1]]) for p in pts]
    ring3, ring2 = list(outline), project(outline)
    if _area(ring2) < 0.0:
        ring3.reverse()
        ring2.reverse()
    for hole in loops[1:]:
        if len(hole) < 3:
            continue
        h3 = [tuple(map(float, p)) for p in hole]
        h2 = project(h3)
        if _area(h2) > 0.0:
            h3.reverse()
            h2.reverse()
        hi = max(range(len(h2)), key=lambda k: h2[k][0])
        order = sorted(range(len(ring2)), key=lambda r: (ring2[r][0] - h2[hi][0]) ** 2 + (ring2[r][1] - h2[hi][1]) ** 2)

        def blocked(a, b):
            return any(_crossing(a, b, poly[i], poly[(i + 1) % len(poly)]) for poly in (ring2, h2)
                       for i in range(len(poly)))
        bridge = next((r for r in order if not blocked(ring2[r], h2[hi])), None)
        if bridge is None:
            return None
        loop = [(hi + k) % len(h3) for k in range(len(h3) + 1)]
        ring3 = ring3[:bridge + 1] + [h3[k] for k in loop] + ring3[bridge:]
        ring2 = ring2[:bridge + 1] + [h2[k] for k in loop] + ring2[bridge:]
    m = len(ring2)
    if m < 3:
        return None
    rem, tris, guard = list(range(m)), [], 0
    while len(rem) > 3 and guard < m * m:
        guard += 1
        clipped = False
        for i in range(len(rem)):
            ia, ib, ic = rem[i - 1], rem[i], rem[(i + 1) % len(rem)]
            a, b, c = ring2[ia], ring2[ib], ring2[ic]
            if _cross(a, b, c) <= 1e-12:
                continue  # reflex or degenerate

            def same(p, q):
                return abs(p[0] - q[0]) < 1e-12 and abs(p[1] - q[1]) < 1e-12
            if any(j not in (ia, ib, ic) and not (same(ring2[j], a) or same(ring2[j], b) or same(ring2[j], c))
                   and _inside(ring2[j], a, b, c) for j in rem):
                continue
            tris.append((ia, ib, ic))
            rem.pop(i)
            clipped = True
            break
        if not clipped:
            break
    tris += [(rem[0], rem[k], rem[k + 1]) for k in range(1, len(rem) - 1)]
    return np.array(ring3, dtype=np.float64), np.array(tris, dtype=np.int64).reshape(-1, 3)
