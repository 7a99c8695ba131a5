"""Accumulation files of distributed renders (src/output/accum.rs): a node
renders a sample range and writes the radiance sums plus per-pixel sample
counts as an OpenEXR image (channels B, G, R, count); `merge` averages any
number of them, as `render merge` does. The file I/O is librtcuda's
(rt_accum_exr_* in include/rt_cuda.h); no GPU is involved."""
import ctypes as C
import os

import numpy as np

from .backend import _check, lib


def write_accum(path, rgbw):
    """(H, W, 4) sums and counts (PtSession.sum_and_weight's layout)."""
    a = np.ascontiguousarray(rgbw, dtype=np.float64)
    h, w = a.shape[:2]
    _check(lib().rt_accum_exr_write(os.fsencode(path), w, h, a.ctypes.data))


def write_accum_exr(path, sum_rgb, count):
    """write_accum_exr (accum.rs:14-46): (H, W, 3) sums, (H, W) counts."""
    s = np.asarray(sum_rgb, dtype=np.float64)
    a = np.concatenate([s, np.asarray(count, dtype=np.float64)[..., None]], axis=2)
    write_accum(path, a)


def accum_size(path):
    w, h = C.c_uint32(), C.c_uint32()
    _check(lib().rt_accum_exr_info(os.fsencode(path), C.byref(w), C.byref(h)))
    return w.value, h.value


def read_accum(path):
    """(H, W, 4) f64: sums and counts of an accumulation file."""
    w, h = accum_size(path)
    a = np.empty((h, w, 4), dtype=np.float64)
    _check(lib().rt_accum_exr_read(os.fsencode(path), w, h, a.ctypes.data))
    return a


def read_accum_exr(path):
    """read_accum_exr (accum.rs:48-85): ((H, W, 3) sums, (H, W) counts)."""
    a = read_accum(path)
    return a[..., :3], a[..., 3]


def merge(files):
    """merge (accum.rs:88-119): the mean image of the files, (H, W, 3) f32."""
    files = [os.fsencode(f) for f in files]
    if not files:
        raise ValueError("merge needs at least one accum file")
    w, h = accum_size(files[0])
    arr = (C.c_char_p * len(files))(*files)
    out = np.empty((h, w, 3), dtype=np.float32)
    _check(lib().rt_accum_merge(arr, len(files), w, h, out.ctypes.data))
    return out


def write_rckp(path, rgbw, passes_done):
    """The Metal backend's checkpoint file (renderer.rs:219-236) of an
    (H, W, 4) accumulator."""
    a = np.ascontiguousarray(rgbw, dtype=np.float64)
    h, w = a.shape[:2]
    _check(lib().rt_rckp_write(os.fsencode(path), w, h, passes_done, a.ctypes.data))
