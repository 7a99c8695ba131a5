"""Radiance .hdr (RGBE) images for dome-light environment maps: what the
reference's EnvMap::load (src/scene/envmap.rs:27-34) reads through the
`image` crate for HDRIs. Flat and run-length ("new-style") scanlines,
"-Y h +X w" orientation (first row at the top); a texel is
mantissa * 2^(exponent - 136), zero when the exponent byte is 0."""
import numpy as np


class HdrError(ValueError):
    pass


def _rle_scanline(data, pos, w):
    """One new-style RLE scanline: 4 channel runs of w bytes each."""
    out = np.empty((4, w), dtype=np.uint8)
    for c in range(4):
        x = 0
        while x < w:
            if pos >= len(data):
                raise HdrError("truncated scanline")
            n = data[pos]
            pos += 1
            if n > 128:
                n -= 128
                if x + n > w or pos >= len(data):
                    raise HdrError("bad run")
                out[c, x:x + n] = data[pos]
                pos += 1
            else:
                if n == 0 or x + n > w or pos + n > len(data):
                    raise HdrError("bad literal run")
                out[c, x:x + n] = np.frombuffer(data, np.uint8, n, pos)
                pos += n
            x += n
    return out.T, pos


def decode_hdr(data):
    """(H, W, 3) float32 radiance from the bytes of a .hdr file."""
    if not (data.startswith(b"#?RADIANCE") or data.startswith(b"#?RGBE")):
        raise HdrError("not a Radiance HDR file")
    pos = 0
    fmt = None
    while True:
        j = data.find(b"\n", pos)
        if j < 0:
            raise HdrError("truncated header")
        line = data[pos:j].strip()
        pos = j + 1
        if not line:
            break
        if line.startswith(b"FORMAT="):
            fmt = line[7:]
    if fmt not in (None, b"32-bit_rle_rgbe"):
        raise HdrError(f"unsupported pixel format {fmt!r}")
    j = data.find(b"\n", pos)
    res = data[pos:j].split()
    pos = j + 1
    if len(res) != 4 or res[0] != b"-Y" or res[2] != b"+X":
        raise HdrError("only -Y h +X w images are supported")
    h, w = int(res[1]), int(res[3])
    rgbe = np.empty((h, w, 4), dtype=np.uint8)
    for y in range(h):
        if 8 <= w < 32768 and pos + 4 <= len(data) and data[pos] == 2 and data[pos + 1] == 2 and \
                (data[pos + 2] << 8 | data[pos + 3]) == w and data[pos + 2] < 128:
            rgbe[y], pos = _rle_scanline(data, pos + 4, w)
        else:
            if pos + 4 * w > len(data):
                raise HdrError("truncated flat scanline")
            rgbe[y] = np.frombuffer(data, np.uint8, 4 * w, pos).reshape(w, 4)
            pos += 4 * w
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(np.float32(1.0), e - 136), 0.0).astype(np.float32)
    return rgbe[..., :3].astype(np.float32) * scale[..., None]


def read_hdr(path):
    with open(path, "rb") as f:
        return decode_hdr(f.read())
