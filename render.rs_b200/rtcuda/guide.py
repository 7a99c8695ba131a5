"""The learned directional proposal through its C ABI (include/rt_guide.h)."""
import ctypes as C

import numpy as np

from .backend import RtError, lib

LEVELS = 16
TABLE_ENTRIES = 1 << 19
MLP_PARAMS = 64 * 48 + 64 * 64 + 64 * 64 + 48 * 64 + 64 * 3 + 48
RECORD = 16
OUTPUTS = 48

# Every entry point declared in include/rt_guide.h.
EXPORTS = ("rt_guide_create", "rt_guide_destroy", "rt_guide_last_error", "rt_guide_train_step",
           "rt_guide_train_step_device", "rt_guide_infer", "rt_guide_infer_device", "rt_guide_infer_mixture",
           "rt_guide_grads",
           "rt_guide_get_params", "rt_guide_set_params", "rt_guide_info", "rt_tc_gemm_selftest")


def _g():
    L = lib()
    if not hasattr(L, "_guide_sigs"):
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.rt_guide_create.argtypes = [vp, vp, u64, C.c_float, C.POINTER(vp)]
        L.rt_guide_destroy.argtypes = [vp]
        L.rt_guide_last_error.restype = C.c_char_p
        L.rt_guide_train_step.argtypes = [vp, vp, u32, vp]
        L.rt_guide_train_step_device.argtypes = [vp, vp, u32, vp, vp]
        L.rt_guide_infer.argtypes = [vp, vp, u32, vp]
        L.rt_guide_infer_device.argtypes = [vp, vp, u32, vp, vp]
        L.rt_guide_infer_mixture.argtypes = [vp, vp, u32, vp]
        L.rt_guide_grads.argtypes = [vp, vp, u32, vp, vp, vp, vp]
        L.rt_guide_get_params.argtypes = [vp, vp, vp]
        L.rt_guide_set_params.argtypes = [vp, vp, vp]
        L.rt_guide_info.argtypes = [vp, vp, vp, vp]
        L.rt_tc_gemm_selftest.argtypes = [vp, vp, C.c_int, C.c_int, vp]
        L._guide_sigs = True
    return L


def _check(rc):
    if rc != 0:
        raise RtError(rc, _g().rt_guide_last_error().decode(errors="replace"))


def tc_gemm_selftest(A_bf16, B_bf16):
    """D[128][N] = A[128][K] B[N][K]^T on the tcgen05 path; bf16 bit patterns in."""
    A = np.ascontiguousarray(A_bf16, dtype=np.uint16)
    B = np.ascontiguousarray(B_bf16, dtype=np.uint16)
    N, K = B.shape
    D = np.zeros((128, N), dtype=np.float32)
    _check(_g().rt_tc_gemm_selftest(A.ctypes.data, B.ctypes.data, N, K, D.ctypes.data))
    return D


class Guide:
    """Hash-grid + MLP -> 8-lobe vMF mixture, trained online with Adam."""

    def __init__(self, lo, hi, seed=1, lr=1e-2):
        lo = np.ascontiguousarray(lo, dtype=np.float32)
        hi = np.ascontiguousarray(hi, dtype=np.float32)
        h = C.c_void_p()
        _check(_g().rt_guide_create(lo.ctypes.data, hi.ctypes.data, seed, lr, C.byref(h)))
        self.h = h

    @classmethod
    def borrow(cls, handle):
        """A view of a network owned elsewhere (a guided session's)."""
        g = cls.__new__(cls)
        g.h = C.c_void_p(handle)
        g._borrowed = True
        return g

    def close(self):
        if getattr(self, "h", None):
            if not getattr(self, "_borrowed", False):
                _g().rt_guide_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def train_step(self, records):
        r = np.ascontiguousarray(records, dtype=np.float32)
        loss = C.c_float()
        _check(_g().rt_guide_train_step(self.h, r.ctypes.data, len(r), C.byref(loss)))
        return loss.value

    def infer(self, records):
        r = np.ascontiguousarray(records, dtype=np.float32)
        out = np.zeros((len(r), OUTPUTS), dtype=np.float32)
        _check(_g().rt_guide_infer(self.h, r.ctypes.data, len(r), out.ctypes.data))
        return out

    def infer_mixture(self, records):
        """The decoded mixture the renderer samples from (48 floats per
        record: 8 x (mu, kappa), 8 weights, 8 log-density offsets A)."""
        r = np.ascontiguousarray(records, dtype=np.float32)
        out = np.zeros((len(r), OUTPUTS), dtype=np.float32)
        _check(_g().rt_guide_infer_mixture(self.h, r.ctypes.data, len(r), out.ctypes.data))
        return out

    def grads(self, records, table=True):
        r = np.ascontiguousarray(records, dtype=np.float32)
        gm = np.zeros(MLP_PARAMS, dtype=np.float32)
        gt = np.zeros(LEVELS * TABLE_ENTRIES * 2, dtype=np.float32) if table else None
        raw = np.zeros((len(r), OUTPUTS), dtype=np.float32)
        loss = C.c_float()
        _check(_g().rt_guide_grads(self.h, r.ctypes.data, len(r), gm.ctypes.data,
                                   gt.ctypes.data if table else None, raw.ctypes.data, C.byref(loss)))
        return raw, loss.value, gm, gt

    def params(self):
        m = np.zeros(MLP_PARAMS, dtype=np.float32)
        t = np.zeros(LEVELS * TABLE_ENTRIES * 2, dtype=np.uint16)
        _check(_g().rt_guide_get_params(self.h, m.ctypes.data, t.ctypes.data))
        return m, t

    def set_params(self, mlp=None, table16=None):
        m = None if mlp is None else np.ascontiguousarray(mlp, dtype=np.float32)
        t = None if table16 is None else np.ascontiguousarray(table16, dtype=np.uint16)
        _check(_g().rt_guide_set_params(self.h, m.ctypes.data if m is not None else None,
                                        t.ctypes.data if t is not None else None))

    def info(self):
        res = np.zeros(16, dtype=np.float32)
        lo = np.zeros(3, dtype=np.float32)
        inv = np.zeros(3, dtype=np.float32)
        _check(_g().rt_guide_info(self.h, res.ctypes.data, lo.ctypes.data, inv.ctypes.data))
        return res, lo, inv


def mixture_pdf(raw, w):
    """Reference decode of raw outputs (numpy, f64): pdf of direction w."""
    raw = np.asarray(raw, dtype=np.float64)
    mu = raw[:40].reshape(8, 5)
    m = mu[:, :3] / np.maximum(np.linalg.norm(mu[:, :3], axis=1, keepdims=True), 1e-8)
    k = np.exp(np.clip(mu[:, 3], -4, 9))
    a = np.exp(mu[:, 4] - mu[:, 4].max())
    a /= a.sum()
    pdf = k / (2 * np.pi * (1 - np.exp(-2 * k))) * np.exp(k * (m @ np.asarray(w) - 1))
    return float((a * pdf).sum())
