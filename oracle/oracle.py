"""ctypes wrapper for the f64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the bench's cpu_baseline / reference legs as the checker and the timed CPU
baseline. The CUDA backend never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class Counters(C.Structure):
    _fields_ = [("node_pops", C.c_uint64), ("tri_tests", C.c_uint64),
                ("inst_tests", C.c_uint64), ("rays", C.c_uint64)]


def build():
    """Compile liboracle.so from the sources in this folder."""
    subprocess.check_call(["make", "-s", "-C", HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, u32p, f64p = C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_double)
        L.oracle_scene_create.restype = vp
        L.oracle_scene_create.argtypes = [vp]
        L.oracle_scene_destroy.argtypes = [vp]
        L.oracle_scene_stats.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.oracle_intersect.argtypes = [vp, vp, C.c_uint64, C.c_int, vp, vp, vp, C.POINTER(Counters), C.c_int]
        L.oracle_render.argtypes = [vp, vp, vp, C.c_uint64, C.c_uint32, C.c_uint32, vp, vp, vp, C.c_int]
        L.oracle_pcg_stream.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, u32p]
        L.oracle_pcg_new_stream.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, u32p]
        L.oracle_bsdf_eval.argtypes = [vp, f64p, f64p, C.c_double, f64p, f64p]
        L.oracle_bsdf_furnace.restype = C.c_double
        L.oracle_bsdf_furnace.argtypes = [vp, f64p, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, f64p]
        L.oracle_light_sample.argtypes = [vp, f64p, C.c_double, u32p, f64p]
        L.oracle_env_eval_pdf.argtypes = [C.c_uint32, C.c_uint32, vp, C.c_uint64, vp, vp, vp]
        L.oracle_env_sample.argtypes = [C.c_uint32, C.c_uint32, vp, C.c_uint64, vp, vp, vp, vp]
        L.oracle_filter_sample.argtypes = [C.c_int, C.c_double, C.c_uint64, vp, vp]
        L.oracle_pattern_eval.argtypes = [vp, C.c_uint32, C.c_uint64, vp, vp]
        L.oracle_intersect_st.argtypes = [vp, C.c_uint64, vp, vp]
        L.oracle_texture_sample.argtypes = [C.c_uint32, C.c_uint32, vp, C.c_int, C.c_uint64, vp, vp]
        L.oracle_ies_eval.argtypes = [C.c_uint32, C.c_uint32, vp, vp, vp, C.c_uint64, vp, vp, vp]
        L.oracle_transmittance.argtypes = [vp, vp, C.c_uint64, vp, C.c_int]
        L.oracle_quadric_intersect.argtypes = [vp, C.c_uint64, vp, vp]
        L.oracle_solve_quartic.argtypes = [vp, vp]
        L.oracle_light_pmf.restype = C.c_double
        L.oracle_light_pmf.argtypes = [vp, f64p, C.c_uint32]
        L.oracle_medium_sample.restype = C.c_uint64
        L.oracle_medium_sample.argtypes = [vp, vp, vp, C.c_double, vp, C.c_uint64, C.c_uint64, C.c_uint64, vp, vp]
        L.oracle_medium_transmittance.argtypes = [vp, vp, vp, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, vp]
        L.oracle_medium_density.argtypes = [vp, C.c_uint64, vp, vp]
        L.oracle_hg_phase.argtypes = [C.c_double, C.c_uint64, vp, vp]
        L.oracle_hg_sample.argtypes = [C.c_double, vp, C.c_uint64, vp, vp]
        L.oracle_sss_medium.argtypes = [vp, vp, vp, vp]
        L.oracle_hair_eval.argtypes = [vp, C.c_uint64, vp, vp, vp]
        L.oracle_hair_sample.argtypes = [vp, vp, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, vp]
        L.oracle_fiber_h.restype = C.c_double
        L.oracle_fiber_h.argtypes = [vp, vp, vp]
        L.oracle_curve_segment.argtypes = [vp, vp, C.c_double, C.c_double, C.c_uint64, vp, vp]
        _lib = L
    return _lib


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _medium_desc(med):
    from rtcuda import abi
    d = abi.RtMediumDesc()
    for key, val in med.items():
        setattr(d, key, abi.c_double3(*val) if isinstance(val, tuple) else val)
    return d


def medium_sample(med, o, d, t_max, beta, pixel, sample, n):
    """n draws of volume.rs sample_distance from one PCG32 stream: (pass
    weight sum, scatter weight sum, scatters)."""
    md = _medium_desc(med)
    o, _ = _f64(o)
    d, _ = _f64(d)
    b, _ = _f64(beta)
    ps, ss = np.zeros(3), np.zeros(3)
    k = lib().oracle_medium_sample(C.byref(md), o.ctypes.data, d.ctypes.data, float(t_max), b.ctypes.data,
                                   int(pixel), int(sample), int(n), ps.ctypes.data, ss.ctypes.data)
    return ps, ss, int(k)


def medium_transmittance(med, o, d, dist, pixel, sample, n):
    """Mean of n volume.rs transmittance estimates (RGB)."""
    md = _medium_desc(med)
    o, _ = _f64(o)
    d, _ = _f64(d)
    out = np.zeros(3)
    lib().oracle_medium_transmittance(C.byref(md), o.ctypes.data, d.ctypes.data, float(dist), int(pixel),
                                      int(sample), int(n), out.ctypes.data)
    return out


def medium_density(med, points):
    md = _medium_desc(med)
    p, _ = _f64(np.reshape(points, (-1, 3)))
    out = np.zeros(len(p))
    lib().oracle_medium_density(C.byref(md), len(p), p.ctypes.data, out.ctypes.data)
    return out


def hg_phase(g, cos_theta):
    c, _ = _f64(np.ravel(cos_theta))
    out = np.zeros(len(c))
    lib().oracle_hg_phase(float(g), len(c), c.ctypes.data, out.ctypes.data)
    return out


def hg_sample(g, wo, u):
    """(wi xyz, pdf) per uniform pair."""
    w, _ = _f64(wo)
    uu, _ = _f64(np.reshape(u, (-1, 2)))
    out = np.zeros((len(uu), 4))
    lib().oracle_hg_sample(float(g), w.ctypes.data, len(uu), uu.ctypes.data, out.ctypes.data)
    return out


def sss_medium(color, dmfp):
    c, _ = _f64(color)
    m, _ = _f64(dmfp)
    sa, ss = np.zeros(3), np.zeros(3)
    lib().oracle_sss_medium(c.ctypes.data, m.ctypes.data, sa.ctypes.data, ss.ctypes.data)
    return sa, ss


def _hair_params(sigma_a, beta_m, beta_n, eta):
    p, _ = _f64(list(np.broadcast_to(np.asarray(sigma_a, float), 3)) + [beta_m, beta_n, eta])
    return p


def hair_eval(params, wo, wi, h):
    """hair::f and hair::pdf for rows of (wo, wi, h); params = (sigma_a,
    beta_m, beta_n, eta)."""
    p = _hair_params(*params)
    wo, wi = np.atleast_2d(wo), np.atleast_2d(wi)
    n = max(len(wo), len(wi))
    q, _ = _f64(np.concatenate([np.broadcast_to(wo, (n, 3)), np.broadcast_to(wi, (n, 3)),
                                np.broadcast_to(np.reshape(h, (-1, 1)), (n, 1))], axis=1))
    f, pdf = np.zeros((n, 3)), np.zeros(n)
    lib().oracle_hair_eval(p.ctypes.data, n, q.ctypes.data, f.ctypes.data, pdf.ctypes.data)
    return f, pdf


def hair_sample(params, wo, h, pixel, sample, n):
    """n draws of hair::sample: (wi, f, pdf), pdf 0 for failed draws."""
    p = _hair_params(*params)
    w, _ = _f64(wo)
    out = np.zeros((n, 7))
    lib().oracle_hair_sample(p.ctypes.data, w.ctypes.data, float(h), int(pixel), int(sample), int(n), out.ctypes.data)
    return out[:, :3], out[:, 3:6], out[:, 6]


def fiber_h(tangent, normal, wo):
    t, _ = _f64(tangent)
    n, _ = _f64(normal)
    w, _ = _f64(wo)
    return lib().oracle_fiber_h(t.ctypes.data, n.ctypes.data, w.ctypes.data)


def curve_segment(p0, p1, v0, v1, origins, directions):
    """One rounded-cone segment against rays: rows of (t or -1, normal,
    tangent, v)."""
    a, _ = _f64(p0)
    b, _ = _f64(p1)
    r, _ = _f64(np.concatenate([np.atleast_2d(origins), np.atleast_2d(directions)], axis=1))
    out = np.zeros((len(r), 8))
    lib().oracle_curve_segment(a.ctypes.data, b.ctypes.data, float(v0), float(v1), len(r), r.ctypes.data,
                               out.ctypes.data)
    return out


def quadric_intersect(desc, origins, directions):
    """One rt_quadric_desc against rays: (n, 10) = t (-1 on a miss), point,
    normal, u, v, st density."""
    r = np.ascontiguousarray(np.hstack([np.atleast_2d(origins), np.atleast_2d(directions)]), dtype=np.float64)
    out = np.empty((len(r), 10))
    lib().oracle_quadric_intersect(C.byref(desc), len(r), r.ctypes.data, out.ctypes.data)
    return out


def solve_quartic(coef):
    c = np.ascontiguousarray(coef, dtype=np.float64)
    roots = np.zeros(4)
    n = lib().oracle_solve_quartic(c.ctypes.data, roots.ctypes.data)
    return roots[:n]


def pcg_stream(pixel, sample, n):
    out = np.zeros(n, dtype=np.uint32)
    lib().oracle_pcg_stream(pixel, sample, n, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out


def pcg_new_stream(seed, stream, n):
    out = np.zeros(n, dtype=np.uint32)
    lib().oracle_pcg_new_stream(seed, stream, n, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out


def bsdf_eval(material_desc, wo, wi, eta):
    f = np.zeros(3)
    pdf = C.c_double()
    _, wop = _f64(wo)
    _, wip = _f64(wi)
    lib().oracle_bsdf_eval(C.byref(material_desc), wop, wip, eta, f.ctypes.data_as(C.POINTER(C.c_double)),
                           C.byref(pdf))
    return f, pdf.value


def bsdf_furnace(material_desc, wo, eta, n, seed=7, stream=11):
    rgb = np.zeros(3)
    _, wop = _f64(wo)
    m = lib().oracle_bsdf_furnace(C.byref(material_desc), wop, eta, n, seed, stream,
                                  rgb.ctypes.data_as(C.POINTER(C.c_double)))
    return m, rgb


class OracleScene:
    """The oracle's view of a scene built from the same ``rt_scene_desc``."""

    def __init__(self, scene):
        self.scene = scene
        self._desc = scene.desc()
        self.h = lib().oracle_scene_create(C.byref(self._desc))
        if not self.h:
            raise RuntimeError("oracle_scene_create failed")

    def close(self):
        if self.h:
            lib().oracle_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self):
        b, t = C.c_uint64(), C.c_uint64()
        lib().oracle_scene_stats(self.h, C.byref(b), C.byref(t))
        return b.value, t.value

    def intersect_st(self, origins, directions):
        """Closest hits of rays: (t or -1, s, t, st density) per ray."""
        r = np.ascontiguousarray(np.hstack([np.atleast_2d(origins), np.atleast_2d(directions)]), dtype=np.float64)
        out = np.empty((len(r), 4))
        lib().oracle_intersect_st(self.h, len(r), r.ctypes.data, out.ctypes.data)
        return out

    def intersect(self, planes, any_hit=False, threads=0):
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        n = planes.shape[1]
        prim = np.zeros(n, dtype=np.uint32)
        inst = np.zeros(n, dtype=np.uint32)
        t = np.zeros(n, dtype=np.float64)
        c = Counters()
        lib().oracle_intersect(self.h, planes.ctypes.data, n, 1 if any_hit else 0, prim.ctypes.data,
                               inst.ctypes.data, t.ctypes.data, C.byref(c), threads)
        return prim, inst, t, c

    def transmittance(self, planes, threads=0):
        """Shadow-ray transmittance (mod.rs:1254-1306) of rays in the
        two-plane layout; (n, 3) RGB."""
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        n = planes.shape[1]
        out = np.zeros((n, 3))
        lib().oracle_transmittance(self.h, planes.ctypes.data, n, out.ctypes.data, threads)
        return out

    def render(self, params, s0, s1, pixels=None, aovs=False, threads=0):
        """Radiance sums over samples [s0, s1) (and AOV sums) for a pixel list;
        the whole image when `pixels` is None."""
        W, H = self.scene.width, self.scene.height
        if pixels is None:
            pixels = np.arange(W * H, dtype=np.uint32)
        pixels = np.ascontiguousarray(pixels, dtype=np.uint32)
        rgb = np.zeros((len(pixels), 3))
        aux = np.zeros((len(pixels), 12)) if aovs else None
        counts = np.zeros(8, dtype=np.uint64)
        rc = lib().oracle_render(self.h, C.byref(params), pixels.ctypes.data, len(pixels), s0, s1, rgb.ctypes.data,
                                 aux.ctypes.data if aovs else None, counts.ctypes.data, threads)
        if rc != 0:
            raise RuntimeError("oracle_render failed")
        return rgb, aux, counts

    def light_sample(self, p, u):
        li, pmf = C.c_uint32(), C.c_double()
        _, pp = _f64(p)
        ok = lib().oracle_light_sample(self.h, pp, u, C.byref(li), C.byref(pmf))
        return (li.value, pmf.value) if ok else None

    def light_pmf(self, p, light):
        _, pp = _f64(p)
        return lib().oracle_light_pmf(self.h, pp, light)


def guide_eval(mlp, table16, res, lo, inv_ext, records, grads=True):
    """f64 network oracle: raw outputs, loss and (optionally) gradients for
    the MLP parameters and the hash table."""
    L = lib()
    if not hasattr(L, "_guide_ready"):
        vp = C.c_void_p
        L.oracle_guide_eval.argtypes = [vp, vp, vp, vp, vp, vp, C.c_uint32, vp, vp, vp, vp]
        L._guide_ready = True
    mlp = np.ascontiguousarray(mlp, dtype=np.float32)
    table16 = np.ascontiguousarray(table16, dtype=np.uint16)
    res = np.ascontiguousarray(res, dtype=np.float32)
    lo = np.ascontiguousarray(lo, dtype=np.float32)
    inv_ext = np.ascontiguousarray(inv_ext, dtype=np.float32)
    rec = np.ascontiguousarray(records, dtype=np.float32)
    n = rec.shape[0]
    raw = np.zeros((n, 48))
    g_mlp = np.zeros(mlp.size) if grads else None
    g_tab = np.zeros(table16.size, dtype=np.float32) if grads else None
    loss = C.c_double()
    L.oracle_guide_eval(mlp.ctypes.data, table16.ctypes.data, res.ctypes.data, lo.ctypes.data, inv_ext.ctypes.data,
                        rec.ctypes.data, n, raw.ctypes.data, g_mlp.ctypes.data if grads else None,
                        g_tab.ctypes.data if grads else None, C.byref(loss))
    return raw, loss.value, g_mlp, g_tab


def env_eval_pdf(env, dirs):
    """envmap.rs eval + pdf for (n, 3) directions on an (H, W, 3) map."""
    e = np.ascontiguousarray(env, dtype=np.float32)
    d = np.ascontiguousarray(dirs, dtype=np.float64)
    rad = np.empty((len(d), 3))
    pdf = np.empty(len(d))
    lib().oracle_env_eval_pdf(e.shape[1], e.shape[0], e.ctypes.data, len(d), d.ctypes.data, rad.ctypes.data,
                               pdf.ctypes.data)
    return rad, pdf


def env_sample(env, uv):
    """envmap.rs sample for (n, 2) uniforms: (dirs, radiance, pdf)."""
    e = np.ascontiguousarray(env, dtype=np.float32)
    u = np.ascontiguousarray(uv, dtype=np.float64)
    dirs, rad, pdf = np.empty((len(u), 3)), np.empty((len(u), 3)), np.empty(len(u))
    lib().oracle_env_sample(e.shape[1], e.shape[0], e.ctypes.data, len(u), u.ctypes.data, dirs.ctypes.data,
                             rad.ctypes.data, pdf.ctypes.data)
    return dirs, rad, pdf


def pattern_eval(scene, node, ctx):
    """pattern.rs eval of `node` of `scene`'s pattern graph at points ctx
    (n, 6) = (s, t, Px, Py, Pz, footprint), or (n, 13) = (s, t, P, N,
    footprint, dst_major, dst_minor); returns (n, 3) RGB."""
    c = np.atleast_2d(np.asarray(ctx, dtype=np.float64))
    if c.shape[1] == 6:
        c = np.hstack([c[:, :5], np.tile([0.0, 0.0, 1.0], (len(c), 1)), c[:, 5:6], np.zeros((len(c), 4))])
    c = np.ascontiguousarray(c)
    out = np.empty((len(c), 3))
    d = scene.desc()
    lib().oracle_pattern_eval(C.addressof(d), int(node), len(c), c.ctypes.data, out.ctypes.data)
    return out


def texture_sample(rgb, queries, wrap=0, ewa=False):
    """texture/cache.rs lookups on the mip chain of `rgb` ((H, W, 3)):
    queries (n, 3) = (s, t, footprint) for `sample`, or (n, 6) = (s, t,
    du, dv) for `sample_ewa` (ewa=True); returns (n, 3) f32."""
    t = np.ascontiguousarray(rgb, dtype=np.float32)
    q = np.atleast_2d(np.asarray(queries, dtype=np.float64))
    full = np.zeros((len(q), 7))
    full[:, :q.shape[1]] = q
    full[:, 6] = 1.0 if ewa else 0.0
    full = np.ascontiguousarray(full)
    out = np.empty((len(q), 3), np.float32)
    lib().oracle_texture_sample(t.shape[1], t.shape[0], t.ctypes.data, int(wrap), len(q), full.ctypes.data,
                                out.ctypes.data)
    return out


def ies_eval(profile, dirs):
    """ies.rs candela_toward and factor of (v_angles, h_angles, candela[h][v])
    toward light-local directions (n, 3); returns (candela, factor)."""
    v, h, c = (np.ascontiguousarray(a, dtype=np.float64) for a in profile)
    d = np.ascontiguousarray(np.atleast_2d(dirs), dtype=np.float64)
    cd, f = np.empty(len(d)), np.empty(len(d))
    lib().oracle_ies_eval(len(v), len(h), v.ctypes.data, h.ctypes.data, c.ctypes.data, len(d), d.ctypes.data,
                          cd.ctypes.data, f.ctypes.data)
    return cd, f


def filter_sample(kind, width, u):
    """camera.rs:36-61 PixelFilter::sample_1d for each uniform in `u`."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.empty(len(u))
    lib().oracle_filter_sample(int(kind), float(width), len(u), u.ctypes.data, out.ctypes.data)
    return out
