"""Radiance .hdr reading for dome-light environment maps
(rtcuda.envmap: the HDRIs the reference's EnvMap::load reads,
src/scene/envmap.rs:27-34), against an RGBE encoder written here."""
import os

import numpy as np
import pytest

from rtcuda.envmap import HdrError, decode_hdr, read_hdr


def _rgbe(img):
    """float (H, W, 3) -> RGBE bytes (H, W, 4), mantissa = c * 256 / 2^e."""
    m = img.max(-1)
    e = np.where(m > 1e-32, np.ceil(np.log2(np.maximum(m, 1e-32)) + 1e-9), 0).astype(np.int32)
    mant = np.where(m[..., None] > 1e-32, np.floor(img * 256.0 / np.exp2(e)[..., None]), 0)
    out = np.zeros(img.shape[:2] + (4,), np.uint8)
    out[..., :3] = np.clip(mant, 0, 255)
    out[..., 3] = np.where(m > 1e-32, e + 128, 0)
    return out


def _encode(rgbe, rle=True):
    h, w = rgbe.shape[:2]
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h):
        if not rle:
            out += rgbe[y].tobytes()
            continue
        out += bytes([2, 2, w >> 8, w & 255])
        for c in range(4):
            row = rgbe[y, :, c]
            x = 0
            while x < w:
                run = 1
                while x + run < w and run < 127 and row[x + run] == row[x]:
                    run += 1
                if run >= 3:
                    out += bytes([128 + run, row[x]])
                    x += run
                else:
                    j = x
                    while j < w and j - x < 128 and not (j + 2 < w and row[j] == row[j + 1] == row[j + 2]):
                        j += 1
                    out += bytes([j - x]) + row[x:j].tobytes()
                    x = j
    return bytes(out)


@pytest.mark.parametrize("rle", [True, False])
def test_decode_matches_rgbe(rle):
    rng = np.random.default_rng(3)
    img = rng.uniform(0, 20, size=(9, 40, 3)).astype(np.float32)
    img[2:5, 5:30] = (100.0, 50.0, 1.0)  # runs
    img[7] = 0.0
    rgbe = _rgbe(img)
    want = rgbe[..., :3].astype(np.float32) * np.where(rgbe[..., 3] > 0, np.exp2(rgbe[..., 3].astype(np.float64) - 136),
                                                        0)[..., None].astype(np.float32)
    got = decode_hdr(_encode(rgbe, rle))
    np.testing.assert_array_equal(got, want)
    assert np.abs(got - img).max() <= img.max() / 64


def test_bad_files():
    with pytest.raises(HdrError):
        decode_hdr(b"P6\n1 1\n255\n000")
    good = _encode(_rgbe(np.ones((4, 16, 3), np.float32)))
    with pytest.raises(HdrError):
        decode_hdr(good[:-5])


SKY = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fixtures", "sky.hdr")


def test_reference_sky_fixture():
    a = read_hdr(SKY)
    assert a.shape == (256, 512, 3) and np.isfinite(a).all() and a.max() > 100
