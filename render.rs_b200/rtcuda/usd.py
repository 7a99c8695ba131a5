"""USD scenes (.usda text) -> rtcuda scenes, as the reference imports them
(src/parser/usd.rs): the stage is translated into RIB requests and fed to
the same scene builder as a RIB file, so USD is a front end, not a second
scene pipeline.

Covered, as in the reference: prim hierarchies (def / over / class) with
xform ops (translate, rotateXYZ, rotateX/Y/Z, scale, transform, in
xformOpOrder or TRS order), Mesh (faceVertexCounts / Indices, points,
per-vertex normals and primvars:st), Sphere and Cube, UsdPreviewSurface
materials bound by ``material:binding``, Distant / Dome / Sphere / Rect
lights, the first Camera (fov from focalLength and horizontalAperture, its
xform chain inverted into the camera transform) and ``upAxis = "Z"``
stages. Composition arcs (references, payloads, variants, inherits) are
skipped with a warning.
"""
import math

from .rib import _Builder

# ---- tokens (usd.rs:39-163) ---------------------------------------------------------------


def _tokens(src):
    """(kind, value) tokens: 'id', 'num', 'str', 'asset', 'path', 'p' (one
    of ( ) [ ] { } , = ;). '#' starts a comment to the end of the line."""
    i, n, out = 0, len(src), []
    while True:
        while i < n:
            if src[i].isspace():
                i += 1
            elif src[i] == "#":
                while i < n and src[i] != "\n":
                    i += 1
            else:
                break
        if i >= n:
            return out
        c = src[i]
        if c in "()[]{},=;":
            out.append(("p", c))
            i += 1
        elif c == '"':
            j = i + 1
            while j < n and src[j] != '"':
                j += 2 if src[j] == "\\" else 1
            out.append(("str", src[i + 1:j]))
            i = j + 1
        elif c in "@<":
            end = "@" if c == "@" else ">"
            j = src.find(end, i + 1)
            j = n if j < 0 else j
            out.append(("asset" if c == "@" else "path", src[i + 1:j]))
            i = j + 1
        elif c.isdigit() or c in "-+.":
            j = i + 1
            while j < n and (src[j].isdigit() or src[j] in ".eE-+"):
                j += 1
            try:
                v = float(src[i:j])
            except ValueError:
                v = 0.0
            out.append(("num", v))
            i = j
        else:
            j = i
            while j < n and (src[j].isalnum() or src[j] in "_:."):
                j += 1
            if j == i:
                i += 1  # an unknown byte
                continue
            out.append(("id", src[i:j]))
            i = j


class _Prim:
    def __init__(self, type_name="", name=""):
        self.type_name, self.name = type_name, name
        self.attrs, self.children = {}, []


class _Parser:
    """usd.rs:165-413: values are ('nums', [..]), ('str', s), ('asset', s),
    ('paths', [..]) or ('tokens', [..])."""

    def __init__(self, text):
        self.t = _tokens(text)
        self.i = 0
        self.warnings = []

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else ("eof", None)

    def next(self):
        tok = self.peek()
        self.i += 1
        return tok

    def skip_parens(self):
        depth = 1
        while depth:
            k, v = self.next()
            if k == "eof":
                raise ValueError("usda: unbalanced metadata parens")
            if k == "p" and v == "(":
                depth += 1
            elif k == "p" and v == ")":
                depth -= 1

    def value(self):
        k, v = self.peek()
        if k == "p" and v == "[":
            self.next()
            nums, strs, paths = [], [], []
            while True:
                k, v = self.next()
                if k == "p" and v == "]":
                    break
                if k == "eof":
                    raise ValueError("usda: unterminated array")
                if k == "num":
                    nums.append(v)
                elif k in ("str", "asset"):
                    strs.append(v)
                elif k == "path":
                    paths.append(v)
                elif k == "p" and v not in ",()":
                    raise ValueError(f"usda: unexpected {v} in array")
            return ("paths", paths) if paths else (("tokens", strs) if strs else ("nums", nums))
        if k == "p" and v == "(":
            self.next()
            nums = []
            while True:
                k, v = self.next()
                if k == "p" and v == ")":
                    return ("nums", nums)
                if k == "eof":
                    raise ValueError("usda: unterminated tuple")
                if k == "num":
                    nums.append(v)
        self.next()
        if k == "num":
            return ("nums", [v])
        if k == "str" or k == "id":
            return ("str", v)
        if k == "asset":
            return ("asset", v)
        if k == "path":
            return ("paths", [v])
        raise ValueError(f"usda: unexpected value token {v!r}")

    def prim_body(self, prim):
        while True:
            k, v = self.next()
            if k == "p" and v == "}":
                return
            if k == "eof":
                raise ValueError("usda: unterminated prim body")
            if k != "id":
                continue
            if v in ("def", "over", "class"):
                prim.children.append(self.prim())
            elif v == "rel":
                k2, name = self.next()
                if k2 != "id":
                    raise ValueError(f"usda: rel name, got {name!r}")
                if self.peek() == ("p", "="):
                    self.next()
                    prim.attrs[name] = self.value()
            else:
                # [qualifiers] type name [= value] [(metadata)]: the last
                # identifier before '=' names the attribute.
                last = v
                while self.peek()[0] == "id":
                    last = self.next()[1]
                if self.peek() == ("p", "="):
                    self.next()
                    val = self.value()
                    if self.peek() == ("p", "("):
                        self.next()
                        self.skip_parens()
                    prim.attrs[last] = val
                elif self.peek() == ("p", "("):
                    self.next()
                    self.skip_parens()

    def prim(self):
        p = _Prim()
        if self.peek()[0] == "id":
            p.type_name = self.next()[1]
        k, v = self.next()
        if k != "str":
            raise ValueError(f"usda: prim name expected, got {v!r}")
        p.name = v
        if self.peek() == ("p", "("):
            self.next()
            self.skip_parens()
            self.warnings.append(f"prim {p.name}: composition metadata ignored (references/variants unsupported)")
        if self.next() != ("p", "{"):
            raise ValueError(f"usda: expected {{ for prim {p.name}")
        self.prim_body(p)
        return p

    def stage(self):
        roots, meta = [], {}
        if self.peek() == ("p", "("):
            self.next()
            depth = 1
            while depth:
                k, v = self.next()
                if k == "eof":
                    raise ValueError("usda: unterminated stage metadata")
                if k == "p" and v == "(":
                    depth += 1
                elif k == "p" and v == ")":
                    depth -= 1
                elif k == "id" and depth == 1 and self.peek() == ("p", "="):
                    self.next()
                    try:
                        meta[v] = self.value()
                    except ValueError:
                        pass
        while True:
            k, v = self.next()
            if k == "eof":
                return roots, meta
            if k == "id" and v in ("def", "over", "class"):
                roots.append(self.prim())


# ---- translation to RIB requests (usd.rs:415-909) ------------------------------------------


def _nums(prim, name):
    v = prim.attrs.get(name)
    return list(v[1]) if v is not None and v[0] == "nums" else None


def _num(prim, name):
    v = _nums(prim, name)
    return v[0] if v else None


def _rot(angle, x, y, z):
    return ("Rotate", [float(angle), float(x), float(y), float(z)])


class _Converter:
    def __init__(self, roots):
        self.roots, self.out, self.warnings = roots, [], []

    def find(self, path):
        parts = path.strip("/").split("/")
        cur = next((p for p in self.roots if p.name == parts[0]), None)
        for part in parts[1:]:
            if cur is None:
                return None
            cur = next((c for c in cur.children if c.name == part), None)
        return cur

    def xform(self, prim):
        order = prim.attrs.get("xformOpOrder")
        if order is not None and order[0] == "tokens":
            ops = list(order[1])
        else:
            ops = [k for k in ("xformOp:translate", "xformOp:rotateXYZ", "xformOp:scale") if k in prim.attrs]
        for op in ops:
            base = op.lstrip("!")
            v = _nums(prim, base)
            if v is None:
                continue
            if base.startswith("xformOp:translate") and len(v) >= 3:
                self.out.append(("Translate", v[:3]))
            elif base.startswith("xformOp:rotateXYZ") and len(v) >= 3:
                # Rx, then Ry, then Rz on points: RIB applies the last first.
                self.out += [_rot(v[2], 0, 0, 1), _rot(v[1], 0, 1, 0), _rot(v[0], 1, 0, 0)]
            elif base.startswith("xformOp:rotateX") and v:
                self.out.append(_rot(v[0], 1, 0, 0))
            elif base.startswith("xformOp:rotateY") and v:
                self.out.append(_rot(v[0], 0, 1, 0))
            elif base.startswith("xformOp:rotateZ") and v:
                self.out.append(_rot(v[0], 0, 0, 1))
            elif base.startswith("xformOp:scale") and len(v) >= 3:
                self.out.append(("Scale", v[:3]))
            elif base.startswith("xformOp:transform") and len(v) >= 16:
                self.out.append(("ConcatTransform", [v[:16]]))
            else:
                self.warnings.append(f"unsupported xform op {base}")

    def material(self, prim):
        """A bound Material's UsdPreviewSurface child -> Bxdf PxrSurface."""
        b = prim.attrs.get("material:binding")
        mat = self.find(b[1][0]) if b is not None and b[0] == "paths" and b[1] else None
        shader = None
        if mat is not None:
            shader = next((c for c in mat.children if c.attrs.get("info:id") == ("str", "UsdPreviewSurface")), None)
        if shader is None:
            return
        diffuse = _nums(shader, "inputs:diffuseColor") or [0.18, 0.18, 0.18]
        rough = _num(shader, "inputs:roughness")
        metallic = _num(shader, "inputs:metallic") or 0.0
        ior = _num(shader, "inputs:ior")
        emissive = _nums(shader, "inputs:emissiveColor") or [0.0, 0.0, 0.0]
        opacity = _num(shader, "inputs:opacity")
        vals = ["PxrSurface", "usd"]
        if metallic > 0.5:
            vals += ["diffuseGain", [0.0], "specularFaceColor", list(diffuse)]
        else:
            vals += ["diffuseGain", [1.0], "diffuseColor", list(diffuse), "specularIor", [1.5 if ior is None else ior]]
        vals += ["specularRoughness", [max(0.5 if rough is None else rough, 0.02)]]
        if any(c > 0.0 for c in emissive):
            vals += ["glowGain", [1.0], "glowColor", list(emissive)]
        if opacity is not None and opacity < 1.0:
            vals += ["presence", [opacity]]
        self.out.append(("Bxdf", vals))

    def light(self, prim):
        kind = {"DistantLight": "PxrDistantLight", "DomeLight": "PxrDomeLight", "SphereLight": "PxrSphereLight",
                "RectLight": "PxrRectLight"}.get(prim.type_name)
        if kind is None:
            return
        inten = _num(prim, "inputs:intensity")
        exp = _num(prim, "inputs:exposure")
        inten = (1.0 if inten is None else inten) * (1.0 if exp is None else 2.0 ** exp)
        vals = [kind, prim.name, "intensity", [inten], "lightColor", _nums(prim, "inputs:color") or [1.0, 1.0, 1.0]]
        extra = {"DistantLight": (("inputs:angle", "angleExtent"),), "SphereLight": (("inputs:radius", "radius"),),
                 "RectLight": (("inputs:width", "width"), ("inputs:height", "height"))}.get(prim.type_name, ())
        for attr, param in extra:
            v = _num(prim, attr)
            if v is not None:
                vals += [param, [v]]
        if prim.type_name == "DomeLight":
            f = prim.attrs.get("inputs:texture:file")
            if f is not None and f[0] == "asset":
                vals += ["lightColorMap", f[1]]
        self.out.append(("Light", vals))

    def geometry(self, prim):
        if prim.type_name == "Mesh":
            counts, idx, pts = (_nums(prim, k) for k in ("faceVertexCounts", "faceVertexIndices", "points"))
            if counts is None or idx is None or pts is None:
                self.warnings.append(f"Mesh {prim.name} missing topology; skipped")
                return
            vals = [counts, idx, "P", pts]
            n = _nums(prim, "normals")
            if n is not None and len(n) == len(pts):
                vals += ["N", n]
            st = _nums(prim, "primvars:st")
            if st is not None and len(st) * 3 == len(pts) * 2:
                vals += ["st", st]
            self.out.append(("PointsPolygons", vals))
        elif prim.type_name == "Sphere":
            r = _num(prim, "radius")
            r = 1.0 if r is None else r
            self.out.append(("Sphere", [r, -r, r, 360.0]))
        elif prim.type_name == "Cube":
            size = _num(prim, "size")
            h = (2.0 if size is None else size) / 2.0
            corners = [(-h, -h, -h), (h, -h, -h), (h, h, -h), (-h, h, -h), (-h, -h, h), (h, -h, h), (h, h, h),
                       (-h, h, h)]
            faces = [0, 3, 2, 1, 4, 5, 6, 7, 0, 1, 5, 4, 2, 3, 7, 6, 1, 2, 6, 5, 0, 4, 7, 3]
            self.out.append(("PointsPolygons", [[4.0] * 6, [float(f) for f in faces], "P",
                                                [c for p in corners for c in p]]))

    def walk(self, prim):
        if prim.type_name in ("Camera", "Material", "Shader"):
            return
        self.out.append(("AttributeBegin", []))
        self.xform(prim)
        self.material(prim)
        self.light(prim)
        self.geometry(prim)
        for c in prim.children:
            self.walk(c)
        self.out.append(("AttributeEnd", []))


def _find_camera(prims, chain):
    for p in prims:
        chain.append(p)
        if p.type_name == "Camera":
            return p
        if _find_camera(p.children, chain) is not None:
            return chain[-1]
        chain.pop()
    return None


def usda_to_requests(text):
    """usda_to_rib: (RIB requests, warnings) for a .usda stage."""
    parser = _Parser(text)
    roots, meta = parser.stage()
    conv = _Converter(roots)
    chain = []
    cam = _find_camera(roots, chain)
    fov = 45.0
    if cam is not None:
        focal = _num(cam, "focalLength")
        aperture = _num(cam, "horizontalAperture")
        focal = 50.0 if focal is None else focal
        aperture = 20.955 if aperture is None else aperture
        fov = 2.0 * math.degrees(math.atan(aperture / (2.0 * focal)))
    out = [("Projection", ["perspective", "fov", [fov]]), ("Scale", [1.0, 1.0, -1.0])]
    # The camera's chain inverted: each prim's ops undone in reverse order,
    # innermost prim first.
    for prim in reversed(chain if cam is not None else []):
        order = prim.attrs.get("xformOpOrder")
        if order is not None and order[0] == "tokens":
            ops = list(reversed(order[1]))
        else:
            ops = [k for k in ("xformOp:scale", "xformOp:rotateXYZ", "xformOp:translate") if k in prim.attrs]
        for op in ops:
            v = _nums(prim, op)
            if v is None:
                continue
            if op.startswith("xformOp:translate") and len(v) >= 3:
                out.append(("Translate", [-v[0], -v[1], -v[2]]))
            elif op.startswith("xformOp:rotateXYZ") and len(v) >= 3:
                out += [_rot(-v[0], 1, 0, 0), _rot(-v[1], 0, 1, 0), _rot(-v[2], 0, 0, 1)]
            elif op.startswith("xformOp:scale") and len(v) >= 3:
                out.append(("Scale", [1.0 / max(x, 1e-9) for x in v[:3]]))
    if meta.get("upAxis") == ("str", "Z"):
        out.append(_rot(-90.0, 1, 0, 0))
    out.append(("WorldBegin", []))
    conv.out = out
    for r in roots:
        conv.walk(r)
    conv.out.append(("WorldEnd", []))
    return conv.out, parser.warnings + conv.warnings


def usda_to_rib(text):
    """The RIB text of a .usda stage's translation (`render catrib
    scene.usda out.rib`)."""
    from .rib import format_rib
    return format_rib(usda_to_requests(text)[0])


def load_usda_string(text, base_dir=None):
    """A RibScene from .usda text (asset paths resolve against base_dir)."""
    reqs, warnings = usda_to_requests(text)
    b = _Builder(base_dir)
    for w in warnings:
        b.warn(w)
    b.run(reqs)
    return b.scene()


def load_usda(path):
    import os
    with open(path, "r", errors="replace") as f:
        return load_usda_string(f.read(), os.path.dirname(os.path.abspath(path)))
