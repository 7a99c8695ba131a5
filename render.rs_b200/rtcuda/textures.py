"""File textures: the reference's tiled, mip-mapped .tex format
(src/texture/tex.rs) and the images a PxrTexture may name.

``write_tex`` / ``read_tex`` follow tex.rs's layout: magic "RTEX", version
1, base width and height, 3 channels, 32-texel tiles, the mip count, then
per mip (width, height, tiles_x, tiles_y, u64 offset) and the tiles of
every mip row-major, each 32 x 32 RGB f32 texels with the partial edge
tiles padded by replicating the last row / column. ``mip_chain`` is the
box chain write_tex builds (2 x 2 average in f32, odd sizes clamp the
second tap) down to 1 x 1; the CUDA backend and the oracle build the same
chain from a base image.

``load_texture`` reads what the reference's cache opens (tex.rs:71-87):
.tex files, Radiance .hdr (linear float) and PNG (8/16-bit, sRGB-decoded);
other formats raise, and the scene reader then binds the reference's
missing-texture colour (magenta).
"""
import struct
import zlib

import numpy as np

TILE = 32
MAGIC = b"RTEX"


class TextureError(ValueError):
    pass


def srgb_to_linear(c):
    """The sRGB transfer function's inverse (IEC 61966-2-1), as tex.rs:60-67."""
    c = np.asarray(c, dtype=np.float32)
    return np.where(c <= np.float32(0.04045), c / np.float32(12.92),
                    ((c + np.float32(0.055)) / np.float32(1.055)) ** np.float32(2.4)).astype(np.float32)


def downsample(img):
    """One 2 x 2 box step (tex.rs:89-110): f32 sum of the four taps in
    (y0 x0, y0 x1, y1 x0, y1 x1) order, times 0.25."""
    h, w = img.shape[:2]
    nh, nw = max(h // 2, 1), max(w // 2, 1)
    y0 = np.minimum(np.arange(nh) * 2, h - 1)
    y1 = np.minimum(np.arange(nh) * 2 + 1, h - 1)
    x0 = np.minimum(np.arange(nw) * 2, w - 1)
    x1 = np.minimum(np.arange(nw) * 2 + 1, w - 1)
    a = img.astype(np.float32)
    s = a[y0][:, x0] + a[y0][:, x1]
    s = s + a[y1][:, x0]
    s = s + a[y1][:, x1]
    return (s * np.float32(0.25)).astype(np.float32)


def mip_chain(img):
    levels = [np.ascontiguousarray(img, dtype=np.float32).reshape(img.shape[0], img.shape[1], 3)]
    while levels[-1].shape[0] > 1 or levels[-1].shape[1] > 1:
        levels.append(downsample(levels[-1]))
    return levels


def write_tex(path, img):
    """Write `img` ((H, W, 3) linear RGB) as a .tex file with its full mip chain."""
    levels = mip_chain(np.asarray(img, dtype=np.float32))
    h, w = levels[0].shape[:2]
    header = 4 + 24 + 24 * len(levels)
    tile_bytes = TILE * TILE * 3 * 4
    infos, off = [], header
    for m in levels:
        tx, ty = -(-m.shape[1] // TILE), -(-m.shape[0] // TILE)
        infos.append((m.shape[1], m.shape[0], tx, ty, off))
        off += tx * ty * tile_bytes
    out = [MAGIC, struct.pack("<6I", 1, w, h, 3, TILE, len(levels))]
    out += [struct.pack("<4IQ", *i) for i in infos]
    for m, (mw, mh, tx, ty, _) in zip(levels, infos):
        # Edge replication: pad to whole tiles with the last row / column.
        ys = np.minimum(np.arange(ty * TILE), mh - 1)
        xs = np.minimum(np.arange(tx * TILE), mw - 1)
        padded = m[ys][:, xs]
        tiles = padded.reshape(ty, TILE, tx, TILE, 3).transpose(0, 2, 1, 3, 4)
        out.append(np.ascontiguousarray(tiles, dtype="<f4").tobytes())
    with open(path, "wb") as f:
        f.write(b"".join(out))


def read_tex_header(data):
    if data[:4] != MAGIC:
        raise TextureError("not a .tex file (bad magic)")
    if len(data) < 28:
        raise TextureError("truncated .tex header")
    version, w, h, ch, tile, n = struct.unpack_from("<6I", data, 4)
    if version != 1:
        raise TextureError(f"unsupported .tex version {version}")
    if ch != 3 or tile != TILE or n > 32 or n == 0:
        raise TextureError("unsupported .tex layout")
    if len(data) < 28 + 24 * n:
        raise TextureError("truncated .tex header")
    mips = [struct.unpack_from("<4IQ", data, 28 + 24 * k) for k in range(n)]
    return w, h, mips


def read_tex_tile(data, mip, tx, ty):
    """One tile of a .tex file's bytes: (32, 32, 3) f32 (tex.rs:222-243)."""
    _, _, mips = read_tex_header(data)
    mw, mh, ntx, nty, off = mips[mip]
    if tx >= ntx or ty >= nty:
        raise TextureError("tile out of range")
    tb = TILE * TILE * 3 * 4
    o = off + (ty * ntx + tx) * tb
    return np.frombuffer(data, "<f4", TILE * TILE * 3, o).reshape(TILE, TILE, 3)


def read_tex(path):
    """The base level of a .tex file as (H, W, 3) f32."""
    with open(path, "rb") as f:
        data = f.read()
    _, _, mips = read_tex_header(data)
    mw, mh, ntx, nty, off = mips[0]
    tb = TILE * TILE * 3 * 4
    if off + ntx * nty * tb > len(data):
        raise TextureError("truncated .tex file")
    tiles = np.frombuffer(data, "<f4", ntx * nty * TILE * TILE * 3, off).reshape(nty, ntx, TILE, TILE, 3)
    return np.ascontiguousarray(tiles.transpose(0, 2, 1, 3, 4).reshape(nty * TILE, ntx * TILE, 3)[:mh, :mw])


def _unfilter(raw, h, stride, bpp):
    """PNG scanline filters 0-4 (ISO/IEC 15948 section 9). None and Up are
    whole-row array operations; Sub, Average and Paeth depend on the byte
    to the left and run per byte on bytearrays."""
    out = np.zeros((h, stride), dtype=np.uint8)
    prev = bytearray(stride)
    pos = 0
    if len(raw) < h * (stride + 1):
        raise TextureError("PNG: truncated image data")
    for y in range(h):
        ftype = raw[pos]
        line = raw[pos + 1:pos + 1 + stride]
        pos += 1 + stride
        if ftype == 0:
            cur = bytearray(line)
        elif ftype == 2:
            cur = bytearray(((np.frombuffer(line, np.uint8).astype(np.uint16) +
                              np.frombuffer(bytes(prev), np.uint8)) & 0xFF).astype(np.uint8).tobytes())
        elif ftype in (1, 3, 4):
            cur = bytearray(line)
            for i in range(stride):
                a = cur[i - bpp] if i >= bpp else 0
                if ftype == 1:
                    p = a
                elif ftype == 3:
                    p = (a + prev[i]) >> 1
                else:
                    b = prev[i]
                    c = prev[i - bpp] if i >= bpp else 0
                    pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                    p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
                cur[i] = (cur[i] + p) & 0xFF
        else:
            raise TextureError(f"PNG: bad filter type {ftype}")
        out[y] = np.frombuffer(bytes(cur), np.uint8)
        prev = cur
    return out


def decode_png(data):
    """Non-interlaced 8/16-bit grey, grey+alpha, RGB or RGBA PNG -> (H, W, 3)
    values in [0, 1] (alpha dropped, grey replicated), not yet linearised."""
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise TextureError("not a PNG file")
    pos, idat, ihdr = 8, [], None
    while pos + 8 <= len(data):
        n, kind = struct.unpack_from(">I4s", data, pos)
        body = data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            if len(body) < 13:
                raise TextureError("PNG: truncated header")
            ihdr = struct.unpack(">IIBBBBB", body[:13])
        elif kind == b"IDAT":
            idat.append(body)
        elif kind == b"IEND":
            break
        pos += 12 + n
    if ihdr is None:
        raise TextureError("PNG without IHDR")
    w, h, depth, ctype, _, _, interlace = ihdr
    chans = {0: 1, 2: 3, 4: 2, 6: 4}.get(ctype)
    if chans is None or depth not in (8, 16) or interlace:
        raise TextureError("PNG: only non-interlaced 8/16-bit grey or RGB(A) images are read")
    bpp = chans * depth // 8
    try:
        raw = zlib.decompress(b"".join(idat))
    except zlib.error as e:
        raise TextureError(f"PNG: {e}") from None
    rows = _unfilter(raw, h, w * bpp, bpp)
    if depth == 16:
        px = rows.reshape(h, w * chans, 2).astype(np.uint32)
        px = ((px[..., 0] << 8) | px[..., 1]).reshape(h, w, chans) / 65535.0
    else:
        px = rows.reshape(h, w, chans) / 255.0
    rgb = px[..., :3] if chans >= 3 else np.repeat(px[..., :1], 3, axis=-1)
    return rgb.astype(np.float32)


def load_texture(path):
    """A texture file as linear RGB f32 (H, W, 3): .tex base level, .hdr as
    stored, PNG sRGB-decoded."""
    low = str(path).lower()
    if low.endswith(".tex"):
        return read_tex(path)
    if low.endswith(".hdr") or low.endswith(".pic"):
        from .envmap import read_hdr
        return np.ascontiguousarray(read_hdr(path), dtype=np.float32)
    if low.endswith(".png"):
        with open(path, "rb") as f:
            return srgb_to_linear(decode_png(f.read()))
    raise TextureError(f"{path}: unsupported texture format (.tex, .hdr and .png are read)")
