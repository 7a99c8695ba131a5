"""The CUDA backend through its C ABI (librtcuda.so, include/rt_cuda.h).

Python mirror of the reference's Metal backend API
(src/raytracer/metal/renderer.rs): ``render_pt`` (:162), ``render_pt_film``
(:180), ``PtSession`` with ``render_samples`` / ``image`` / ``sum_and_weight``
(:275-490), checkpointing (:219-254) and ``intersect_probe`` (:813-877).
Errors raise ``RtError`` with the library's message, as the reference's
functions return ``anyhow`` errors.

There is no CPU fallback: if librtcuda.so is missing or cannot be loaded,
every call raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "librtcuda.so")

RT_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory", -4: "device overrun",
          -5: "I/O error", -6: "checkpoint mismatch"}

# Every entry point declared in include/rt_cuda.h.
EXPORTS = ("rt_session_create", "rt_session_destroy", "rt_last_error", "rt_render_samples", "rt_reset",
           "rt_read_accum", "rt_read_image", "rt_read_aux", "rt_checkpoint_save", "rt_checkpoint_load",
           "rt_intersect_batch", "rt_intersect_batch_device", "rt_get_stats", "rt_session_stream",
           "rt_bsdf_furnace", "rt_hair_eval", "rt_hair_sample", "rt_intersect_batch_noalloc", "rt_session_guide", "rt_set_adaptive",
           "rt_average_spp", "rt_checkpoint_save_rckp", "rt_rckp_write", "rt_accum_exr_write",
           "rt_accum_exr_info", "rt_accum_exr_read", "rt_accum_merge", "rt_read_film", "rt_denoise",
           "rt_denoise_film", "rt_film_exr_write", "rt_pcg_streams", "rt_light_sample_batch",
           "rt_light_pmf_batch", "rt_transmittance_batch", "rt_set_limits")


class RtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


class RtStats(C.Structure):
    _fields_ = [("blas_nodes", C.c_uint64), ("tlas_nodes", C.c_uint64), ("triangles", C.c_uint64),
                ("device_bytes", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("samples", C.c_uint64), ("kernel_launches", C.c_uint64), ("extend_ms", C.c_double),
                ("shadow_ms", C.c_double), ("shade_ms", C.c_double), ("total_ms", C.c_double),
                ("guide_steps", C.c_uint64), ("guide_records", C.c_uint64), ("guide_loss", C.c_double),
                ("slabs", C.c_uint64), ("waves", C.c_uint64)]


_lib = None


def build():
    """Compile librtcuda.so for sm_100a (nvcc cross-compiles without a GPU)."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", PKG])


def lib():
    """Load librtcuda.so; raises when it is absent (no silent fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RtError(-2, f"{LIB_PATH} is missing: build it with `make -C {PKG}`")
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
        L.rt_session_create.argtypes = [vp, vp, C.POINTER(vp)]
        L.rt_session_destroy.argtypes = [vp]
        L.rt_last_error.restype = C.c_char_p
        L.rt_render_samples.argtypes = [vp, u32, u32]
        L.rt_reset.argtypes = [vp]
        L.rt_read_accum.argtypes = [vp, vp]
        L.rt_read_image.argtypes = [vp, vp]
        L.rt_read_aux.argtypes = [vp, vp]
        L.rt_checkpoint_save.argtypes = [vp, C.c_char_p]
        L.rt_checkpoint_load.argtypes = [vp, C.c_char_p, C.POINTER(u32)]
        L.rt_intersect_batch.argtypes = [vp, vp, u64, i32, vp, vp, vp]
        L.rt_intersect_batch_device.argtypes = [vp, vp, u64, i32, vp, vp, vp, vp]
        L.rt_get_stats.argtypes = [vp, C.POINTER(RtStats)]
        L.rt_bsdf_furnace.argtypes = [vp, vp, C.c_double, u64, u64, vp]
        L.rt_session_stream.restype = vp
        L.rt_session_stream.argtypes = [vp]
        L.rt_session_guide.restype = vp
        L.rt_session_guide.argtypes = [vp]
        L.rt_set_adaptive.argtypes = [vp, C.c_double]
        L.rt_average_spp.argtypes = [vp, C.POINTER(C.c_double)]
        L.rt_checkpoint_save_rckp.argtypes = [vp, C.c_char_p]
        L.rt_rckp_write.argtypes = [C.c_char_p, u32, u32, u32, vp]
        L.rt_accum_exr_write.argtypes = [C.c_char_p, u32, u32, vp]
        L.rt_accum_exr_info.argtypes = [C.c_char_p, C.POINTER(u32), C.POINTER(u32)]
        L.rt_accum_exr_read.argtypes = [C.c_char_p, u32, u32, vp]
        L.rt_accum_merge.argtypes = [C.POINTER(C.c_char_p), u32, u32, u32, vp]
        L.rt_read_film.argtypes = [vp, vp]
        L.rt_denoise.argtypes = [vp, vp]
        L.rt_denoise_film.argtypes = [vp, u32, u32, vp]
        L.rt_film_exr_write.argtypes = [C.c_char_p, u32, u32, vp, C.c_char_p]
        L.rt_pcg_streams.argtypes = [vp, vp, u32, u32, vp]
        L.rt_hair_eval.argtypes = [vp, C.c_uint64, vp, vp, vp]
        L.rt_hair_sample.argtypes = [vp, vp, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, vp]
        L.rt_light_sample_batch.argtypes = [vp, vp, vp, u32, vp, vp]
        L.rt_light_pmf_batch.argtypes = [vp, vp, vp, u32, vp]
        L.rt_transmittance_batch.argtypes = [vp, vp, u64, vp]
        L.rt_set_limits.argtypes = [vp, u32, u32]
        _lib = L
    return _lib


def _check(rc):
    if rc != RT_OK:
        raise RtError(rc, lib().rt_last_error().decode(errors="replace"))


def pcg_streams(pixels, samples, n):
    """(m, n) u32 draws of the device PCG32 of each (pixel, sample) pair."""
    px = np.ascontiguousarray(pixels, dtype=np.uint64)
    sm = np.ascontiguousarray(samples, dtype=np.uint64)
    out = np.empty((len(px), n), np.uint32)
    _check(lib().rt_pcg_streams(px.ctypes.data, sm.ctypes.data, len(px), n, out.ctypes.data))
    return out


def _hair_params(params):
    sa, bm, bn, eta = params
    return np.ascontiguousarray(list(np.broadcast_to(np.asarray(sa, float), 3)) + [bm, bn, eta], dtype=np.float64)


def hair_eval(params, wo, wi, h):
    """Device hair::f and hair::pdf (rt_hair_eval) for rows of (wo, wi, h)
    in the fiber frame; params = (sigma_a, beta_m, beta_n, eta)."""
    p = _hair_params(params)
    wo, wi = np.atleast_2d(wo), np.atleast_2d(wi)
    n = max(len(wo), len(wi))
    q = np.ascontiguousarray(np.concatenate([np.broadcast_to(wo, (n, 3)), np.broadcast_to(wi, (n, 3)),
                                             np.broadcast_to(np.reshape(h, (-1, 1)), (n, 1))], axis=1),
                             dtype=np.float32)
    f, pdf = np.empty((n, 3), np.float32), np.empty(n, np.float32)
    _check(lib().rt_hair_eval(p.ctypes.data, n, q.ctypes.data, f.ctypes.data, pdf.ctypes.data))
    return f, pdf


def hair_sample(params, wo, h, pixel, sample, n):
    """n device hair samples (rt_hair_sample): (wi, f, pdf)."""
    p = _hair_params(params)
    w = np.ascontiguousarray(wo, dtype=np.float64)
    out = np.empty((n, 7), np.float32)
    _check(lib().rt_hair_sample(p.ctypes.data, w.ctypes.data, C.c_double(h), C.c_uint64(pixel), C.c_uint64(sample),
                                C.c_uint64(n), out.ctypes.data))
    return out[:, :3], out[:, 3:6], out[:, 6]


class PtSession:
    """Persistent GPU path-tracing session (renderer.rs:262-490): uploaded
    scene + f64 accumulation state, adding samples incrementally."""

    def __init__(self, scene, params=None, **kw):
        self.scene = scene
        self.params = params if params is not None else abi.make_params(**kw)
        self.width, self.height = scene.width, scene.height
        self._desc = scene.desc()
        h = C.c_void_p()
        _check(lib().rt_session_create(C.byref(self._desc), C.byref(self.params), C.byref(h)))
        self.h = h
        self.samples_done = 0

    def close(self):
        if getattr(self, "h", None):
            lib().rt_session_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render_samples(self, start, count):
        _check(lib().rt_render_samples(self.h, start, count))
        self.samples_done = max(self.samples_done, start + count)

    def reset(self):
        _check(lib().rt_reset(self.h))
        self.samples_done = 0

    def set_adaptive(self, tol):
        """Adaptive stopping (WfSession::set_adaptive): 0 turns it off."""
        _check(lib().rt_set_adaptive(self.h, float(tol)))

    def average_spp(self):
        """Samples per pixel actually taken (WfSession::average_spp)."""
        v = C.c_double()
        _check(lib().rt_average_spp(self.h, C.byref(v)))
        return v.value

    def sum_and_weight(self):
        """(H, W, 4) f64: radiance sums and the sample weight."""
        a = np.empty((self.height, self.width, 4), dtype=np.float64)
        _check(lib().rt_read_accum(self.h, a.ctypes.data))
        return a

    def image(self):
        a = np.empty((self.height, self.width, 3), dtype=np.float32)
        _check(lib().rt_read_image(self.h, a.ctypes.data))
        return a

    def aux(self):
        a = np.empty((self.height, self.width, 12), dtype=np.float32)
        _check(lib().rt_read_aux(self.h, a.ctypes.data))
        return a

    def checkpoint_save(self, path):
        _check(lib().rt_checkpoint_save(self.h, os.fsencode(path)))

    def film_array(self):
        """(H, W, 18) f32 film decoded on the device (RT_FILM_* layout)."""
        a = np.empty((self.height, self.width, FILM_FLOATS), dtype=np.float32)
        _check(lib().rt_read_film(self.h, a.ctypes.data))
        return a

    def film(self):
        """The AOV film as a dict of layers (src/output/film.rs: Film)."""
        return film_layers(self.film_array())

    def denoise(self):
        """output::denoise of this session's film (needs aovs=True), (H, W, 3)."""
        a = np.empty((self.height, self.width, 3), dtype=np.float32)
        _check(lib().rt_denoise(self.h, a.ctypes.data))
        return a

    def checkpoint_save_rckp(self, path):
        """The Metal backend's f32 checkpoint format (renderer.rs:219-236)."""
        _check(lib().rt_checkpoint_save_rckp(self.h, os.fsencode(path)))

    def write_accum_exr(self, path):
        """This session's sums and sample counts as an accumulation EXR
        (the --sample-range output, src/main.rs:363-403)."""
        from .accum import write_accum
        write_accum(path, self.sum_and_weight())

    def checkpoint_load(self, path):
        done = C.c_uint32()
        _check(lib().rt_checkpoint_load(self.h, os.fsencode(path), C.byref(done)))
        self.samples_done = done.value
        return done.value

    def intersect(self, planes, any_hit=False):
        """Ray batch (see triangle_cloud_rays for the plane layout)."""
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        n = planes.shape[1]
        prim = np.empty(n, dtype=np.uint32)
        inst = np.empty(n, dtype=np.uint32)
        t = np.empty(n, dtype=np.float32)
        _check(lib().rt_intersect_batch(self.h, planes.ctypes.data, n, 1 if any_hit else 0, prim.ctypes.data,
                                        inst.ctypes.data, t.ctypes.data))
        return (prim.astype(bool), None, None) if any_hit else (prim, inst, t)

    def intersect_device(self, planes_ptr, n, any_hit, prim_ptr, inst_ptr=None, t_ptr=None, stream=None):
        """Device-pointer ray batch, enqueued without a host sync."""
        _check(lib().rt_intersect_batch_device(self.h, planes_ptr, n, 1 if any_hit else 0, prim_ptr, inst_ptr,
                                               t_ptr, stream))

    def set_limits(self, max_trav_steps=0, wait_polls=0):
        """Limits of the device's bounded loops (0 = defaults)."""
        _check(lib().rt_set_limits(self.h, max_trav_steps, wait_polls))

    def light_sample(self, points, u):
        """Device light-BVH picks at (m, 3) points with (m,) uniforms:
        (light indices, pick probabilities)."""
        p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        uu = np.ascontiguousarray(u, dtype=np.float32)
        light = np.empty(len(p), np.uint32)
        pmf = np.empty(len(p), np.float32)
        _check(lib().rt_light_sample_batch(self.h, p.ctypes.data, uu.ctypes.data, len(p), light.ctypes.data,
                                           pmf.ctypes.data))
        return light, pmf

    def light_pmf(self, points, lights):
        """Device pick probability of lights[i] at points[i]."""
        p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        li = np.ascontiguousarray(lights, dtype=np.uint32)
        pmf = np.empty(len(p), np.float32)
        _check(lib().rt_light_pmf_batch(self.h, p.ctypes.data, li.ctypes.data, len(p), pmf.ctypes.data))
        return pmf

    def transmittance(self, planes):
        """Shadow-ray transmittance of rays in the two-plane layout."""
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        n = planes.shape[1]
        out = np.empty(n, np.float32)
        _check(lib().rt_transmittance_batch(self.h, planes.ctypes.data, n, out.ctypes.data))
        return out

    def stats(self):
        s = RtStats()
        _check(lib().rt_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in RtStats._fields_}

    def stream(self):
        return lib().rt_session_stream(self.h)

    def guide(self):
        """The session's trained proposal network (rtcuda.guide.Guide view,
        owned by the session), or None when the session is not guided."""
        from .guide import Guide
        h = lib().rt_session_guide(self.h)
        return Guide.borrow(h) if h else None


def bsdf_furnace(material, wo, eta, n, seed=1):
    """GPU white-furnace estimate (see rt_bsdf_furnace): (mean lum weight, rgb)."""
    m = abi.RtMaterialDesc()
    for key, val in material.items():
        setattr(m, key, abi.c_double3(*val) if isinstance(val, tuple) else val)
    w = np.ascontiguousarray(wo, dtype=np.float64)
    out = np.zeros(4)
    _check(lib().rt_bsdf_furnace(C.byref(m), w.ctypes.data, eta, n, seed, out.ctypes.data))
    return out[0], out[1:]


def render_pt(scene, spp, **kw):
    """metal::render_pt (renderer.rs:162): beauty image after `spp` samples."""
    with PtSession(scene, **kw) as s:
        s.render_samples(0, spp)
        return s.image()


def render_pt_checkpointed(scene, spp, checkpoint=None, every=4, **kw):
    """metal::render_pt_checkpointed (renderer.rs:170-177): resumes from and
    writes `checkpoint` every `every` samples (atomic tmp + rename)."""
    with PtSession(scene, **kw) as s:
        done = 0
        if checkpoint and os.path.exists(checkpoint):
            try:
                done = s.checkpoint_load(checkpoint)
            except RtError:
                done = 0
        while done < spp:
            n = min(every, spp - done)
            s.render_samples(done, n)
            done += n
            if checkpoint:
                s.checkpoint_save(checkpoint)
        return s.image()


FILM_FLOATS = 18
FILM_LAYERS = {"beauty": (0, 3), "diffuse": (3, 3), "specular": (6, 3), "albedo": (9, 3), "normal": (12, 3),
               "depth": (15, 1), "id": (16, 2)}


def film_layers(arr):
    """Dict of layers from an (H, W, 18) film array."""
    return {k: arr[..., o:o + n] for k, (o, n) in FILM_LAYERS.items()}


def film_array(film):
    """(H, W, 18) f32 film array from a dict of layers."""
    h, w = film["beauty"].shape[:2]
    a = np.zeros((h, w, FILM_FLOATS), dtype=np.float32)
    for k, (o, n) in FILM_LAYERS.items():
        a[..., o:o + n] = np.asarray(film[k], dtype=np.float32).reshape(h, w, -1)[..., :n]
    return a


def denoise_film(film):
    """output::denoise (src/output/denoise.rs:28-139) on the GPU for a film
    dict or (H, W, 18) array; returns the (H, W, 3) beauty."""
    a = np.ascontiguousarray(film if isinstance(film, np.ndarray) else film_array(film), dtype=np.float32)
    h, w = a.shape[:2]
    out = np.empty((h, w, 3), dtype=np.float32)
    _check(lib().rt_denoise_film(a.ctypes.data, w, h, out.ctypes.data))
    return out


def write_multilayer_exr(film, path, manifest=None):
    """write_multilayer_exr (src/output/multilayer.rs): manifest {id: name}."""
    a = np.ascontiguousarray(film if isinstance(film, np.ndarray) else film_array(film), dtype=np.float32)
    h, w = a.shape[:2]
    m = ";".join(f"{k}:{v}" for k, v in sorted(manifest.items())).encode() if manifest else None
    _check(lib().rt_film_exr_write(os.fsencode(path), w, h, a.ctypes.data, m))


def decode_film(beauty, aux, spp):
    """render_pt_film's AOV decode (renderer.rs:180-217)."""
    inv = 1.0 / spp
    hits = aux[..., 11:12]
    film = {
        "beauty": beauty,
        "albedo": aux[..., 0:3] * inv,
        "normal": aux[..., 3:6] * inv,
        "depth": np.where(hits > 0, aux[..., 6:7] / np.maximum(hits, 1), 0.0),
        "id": np.concatenate([aux[..., 7:8], np.minimum(hits * inv, 1.0)], axis=-1),
        "diffuse": aux[..., 8:11] * inv,
    }
    film["specular"] = np.maximum(beauty - film["diffuse"], 0.0)
    return film


def render_pt_film(scene, spp, **kw):
    """metal::render_pt_film (renderer.rs:180-217): beauty + AOVs."""
    kw["aovs"] = True
    with PtSession(scene, **kw) as s:
        s.render_samples(0, spp)
        return decode_film(s.image(), s.aux(), spp)


def intersect_probe(scene, planes, any_hit=False, **kw):
    """Ray batch against a scene (renderer.rs:813-877 for primitives)."""
    with PtSession(scene, **kw) as s:
        return s.intersect(planes, any_hit)
