"""The film post-pass formats and the denoiser's oracle, on the CPU:
the reference's denoise test (src/output/denoise.rs:141-208) pins the f64
oracle the GPU denoiser is checked against, and the multilayer EXR writer
is read back as the reference's own test does (src/output/multilayer.rs)."""
import os
import struct
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import denoise_oracle  # noqa: E402  (the checker)

from rtcuda.backend import FILM_LAYERS, film_array, write_multilayer_exr  # noqa: E402


def noisy_halves_film(w=64, h=64):
    """The reference test's film: left half bright (id 1), right half dark
    (id 2), uniform noise from a 64-bit LCG, flat normal, depth 5."""
    state = 42
    beauty = np.zeros((h, w, 3))
    albedo = np.zeros((h, w, 3))
    ids = np.zeros((h, w, 2))
    for y in range(h):
        for x in range(w):
            left = x < w // 2
            base = 0.8 if left else 0.1
            state = (state * 6364136223846793005 + 1) % (1 << 64)
            noise = ((state >> 33) / float(1 << 31) - 0.5) * 0.4
            beauty[y, x] = max(base + noise, 0.0)
            albedo[y, x] = base
            ids[y, x] = (1.0 if left else 2.0, 1.0)
    normal = np.zeros((h, w, 3))
    normal[..., 2] = 1.0
    return {"beauty": beauty, "diffuse": beauty.copy(), "specular": np.zeros((h, w, 3)), "albedo": albedo,
            "normal": normal, "depth": np.full((h, w, 1), 5.0), "id": ids}


def check_reference_denoise_properties(film, out):
    h, w = out.shape[:2]
    a = np.asarray(film["beauty"])[8:h - 8, 8:w // 2 - 8, 0]
    b = out[8:h - 8, 8:w // 2 - 8, 0]
    assert b.var() < a.var() * 0.05, (a.var(), b.var())
    assert abs(b.mean() - a.mean()) < 0.02
    assert out[h // 2, w // 2 - 1, 0] - out[h // 2, w // 2, 0] > 0.5


def test_oracle_passes_the_reference_denoise_test():
    film = noisy_halves_film()
    check_reference_denoise_properties(film, denoise_oracle.denoise(film))


def _read_exr_header(b):
    assert struct.unpack("<II", b[:8]) == (20000630, 2)
    p, attrs = 8, {}
    while b[p] != 0:
        n = b[p:b.index(b"\0", p)].decode()
        p += len(n) + 1
        t = b[p:b.index(b"\0", p)].decode()
        p += len(t) + 1
        sz = struct.unpack("<I", b[p:p + 4])[0]
        attrs[n] = (t, b[p + 4:p + 4 + sz])
        p += 4 + sz
    return attrs, p + 1


def test_multilayer_exr_round_trip(tmp_path):
    # multilayer.rs tests: an 8 x 6 film of gradients with an id manifest.
    w, h = 8, 6
    grad = lambda f: np.stack(np.broadcast_arrays(np.arange(w)[None, :] * f, np.arange(h)[:, None] * f,
                                                  np.full((h, w), 0.25)), -1)
    film = {"beauty": grad(0.1), "diffuse": grad(0.05), "specular": grad(0.05), "albedo": grad(0.08),
            "normal": grad(0.02), "depth": grad(1.0)[..., :1], "id": grad(1.0)[..., :2]}
    path = tmp_path / "film.exr"
    write_multilayer_exr(film, path, {1: "hero", 2: "floor"})
    b = path.read_bytes()
    attrs, p = _read_exr_header(b)
    chl = attrs["channels"][1]
    names, q = [], 0
    while chl[q] != 0:
        n = chl[q:chl.index(b"\0", q)].decode()
        names.append(n)
        q += len(n) + 1 + 16
    assert names == sorted(names) and len(names) == 18
    assert set(names) == {"R", "G", "B", "diffuse.R", "diffuse.G", "diffuse.B", "specular.R", "specular.G",
                          "specular.B", "albedo.R", "albedo.G", "albedo.B", "N.X", "N.Y", "N.Z", "depth.Z",
                          "id.x", "id.coverage"}
    assert attrs["name"][1] == b"rgba"
    assert attrs["render_rs/manifest"][1] == b"1:hero;2:floor"
    offs = struct.unpack(f"<{h}Q", b[p:p + 8 * h])
    arr = film_array(film)
    src = {"R": ("beauty", 0), "G": ("beauty", 1), "B": ("beauty", 2), "N.X": ("normal", 0), "N.Y": ("normal", 1),
           "N.Z": ("normal", 2), "depth.Z": ("depth", 0), "id.x": ("id", 0), "id.coverage": ("id", 1)}
    for n in names:
        if n.split(".")[0] in ("diffuse", "specular", "albedo"):
            src[n] = (n.split(".")[0], "RGB".index(n.split(".")[1]))
    for y in range(h):
        o = offs[y]
        assert struct.unpack("<ii", b[o:o + 8]) == (y, 4 * 18 * w)
        row = np.frombuffer(b[o + 8:o + 8 + 4 * 18 * w], "<f4").reshape(18, w)
        for k, n in enumerate(names):
            layer, c = src[n]
            np.testing.assert_array_equal(row[k], arr[y, :, FILM_LAYERS[layer][0] + c])
