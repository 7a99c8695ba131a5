"""Accumulation files (src/output/accum.rs) and the Metal checkpoint format
(src/raytracer/metal/renderer.rs:219-254) through librtcuda's host-side
readers and writers; no GPU needed. The merge known-answer case is the
reference's own test (accum.rs: accum_round_trip_and_merge). Compressed and
tiled inputs are produced by the small OpenEXR encoder below (the format's
published RLE / ZIP block coding: even/odd byte split, byte-delta predictor,
then run-length or zlib), standing in for files of other writers."""
import struct
import zlib

import numpy as np
import pytest

from rtcuda import RtError, accum


def _ref_images(w=8, h=6):
    a = np.array([[[x * 4.0, y * 4.0, 1.0 * 4.0, 4.0] for x in range(w)] for y in range(h)])
    b = np.array([[[x * 4.0, y * 4.0, 3.0 * 4.0, 4.0] for x in range(w)] for y in range(h)])
    return a, b


def test_reference_round_trip_and_merge(tmp_path):
    a, b = _ref_images()
    pa, pb = tmp_path / "a.exr", tmp_path / "b.exr"
    accum.write_accum_exr(pa, a[..., :3], a[..., 3])
    accum.write_accum_exr(pb, b[..., :3], b[..., 3])
    merged = accum.merge([pa, pb])
    expect = (a[3, 5, :3] + b[3, 5, :3]) / 8.0  # mean = (a + b) / 8 samples
    assert np.linalg.norm(merged[3, 5] - expect) < 1e-5
    np.testing.assert_allclose(merged, (a[..., :3] + b[..., :3]) / 8.0, rtol=0, atol=1e-6)
    s, c = accum.read_accum_exr(pa)
    np.testing.assert_array_equal(s, a[..., :3])
    np.testing.assert_array_equal(c, a[..., 3])


def test_round_trip_is_f32_exact_and_zero_counts_merge_to_black(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.uniform(0, 1e3, size=(13, 17, 4)).astype(np.float32).astype(np.float64)
    a[2, 3, 3] = 0.0
    p = tmp_path / "x.exr"
    accum.write_accum(p, a)
    assert accum.accum_size(p) == (17, 13)
    np.testing.assert_array_equal(accum.read_accum(p), a)
    m = accum.merge([p])
    assert (m[2, 3] == 0).all()
    np.testing.assert_allclose(m[5, 6], a[5, 6, :3] / a[5, 6, 3], rtol=1e-6)


# ---- an independent OpenEXR encoder for compressed / tiled inputs ------------------------------
def _attr(name, typ, data):
    return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<I", len(data)) + data


def _chlist(chans):
    out = b""
    for name, typ in chans:
        out += name.encode() + b"\0" + struct.pack("<iB3xii", typ, 0, 1, 1)
    return out + b"\0"


def _predict(raw):
    half = (len(raw) + 1) // 2
    t = bytearray(len(raw))
    t[:half] = raw[0::2]
    t[half:] = raw[1::2]
    out = bytearray(t)
    for i in range(len(t) - 1, 0, -1):
        out[i] = (t[i] - t[i - 1] + 128 + 256) & 0xFF
    return bytes(out)


def _rle(data):
    out, i, n = bytearray(), 0, len(data)
    while i < n:
        run = 1
        while i + run < n and run < 128 and data[i + run] == data[i]:
            run += 1
        if run >= 3:
            out += struct.pack("b", run - 1) + data[i:i + 1]
            i += run
        else:
            j = i
            while j < n and j - i < 127 and not (j + 2 < n and data[j] == data[j + 1] == data[j + 2]):
                j += 1
            out += struct.pack("b", -(j - i)) + data[i:j]
            i = j
    return bytes(out)


def _encode(raw, comp):
    if comp == 0:
        return raw
    body = _rle(_predict(raw)) if comp == 1 else zlib.compress(_predict(raw))
    return body if len(body) < len(raw) else raw


def _exr(img, comp, tiles=None, half=False, order=("B", "G", "R", "count")):
    """img: (H, W, 4) as (R, G, B, count)."""
    h, w = img.shape[:2]
    idx = {"R": 0, "G": 1, "B": 2, "count": 3, "A": 3}
    chans = sorted(order)
    typ = 1 if half else 2
    hdr = _attr("channels", "chlist", _chlist([(c, typ) for c in chans]))
    hdr += _attr("compression", "compression", bytes([comp]))
    box = struct.pack("<4i", 0, 0, w - 1, h - 1)
    hdr += _attr("dataWindow", "box2i", box) + _attr("displayWindow", "box2i", box)
    hdr += _attr("lineOrder", "lineOrder", b"\0")
    hdr += _attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    hdr += _attr("screenWindowCenter", "v2f", struct.pack("<2f", 0, 0))
    hdr += _attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
    if tiles:
        hdr += _attr("tiles", "tiledesc", struct.pack("<IIB", tiles, tiles, 0))
    hdr += b"\0"
    dt = np.float16 if half else np.float32

    def block(x0, y0, bw, bh):
        raw = b""
        for y in range(y0, y0 + bh):
            for c in chans:
                raw += img[y, x0:x0 + bw, idx[c]].astype(dt).astype("<" + np.dtype(dt).str[1:]).tobytes()
        return _encode(raw, comp)

    chunks = []
    if tiles:
        for ty in range((h + tiles - 1) // tiles):
            for tx in range((w + tiles - 1) // tiles):
                x0, y0 = tx * tiles, ty * tiles
                data = block(x0, y0, min(tiles, w - x0), min(tiles, h - y0))
                chunks.append(struct.pack("<4ii", tx, ty, 0, 0, len(data)) + data)
    else:
        lines = 16 if comp == 3 else 1
        for y0 in range(0, h, lines):
            data = block(0, y0, w, min(lines, h - y0))
            chunks.append(struct.pack("<ii", y0, len(data)) + data)
    version = 2 | (0x200 if tiles else 0)
    head = struct.pack("<II", 20000630, version) + hdr
    off = len(head) + 8 * len(chunks)
    table = b""
    for c in chunks:
        table += struct.pack("<Q", off)
        off += len(c)
    return head + table + b"".join(chunks)


@pytest.mark.parametrize("comp,tiles,half", [(0, None, False), (1, None, False), (2, None, False),
                                              (3, None, False), (1, 64, False), (3, 16, False),
                                              (0, None, True), (1, 64, True)])
def test_reads_compressed_tiled_and_half_files(tmp_path, comp, tiles, half):
    rng = np.random.default_rng(comp * 7 + (tiles or 0))
    h, w = 70, 83  # ragged against 16-line and 64-pixel blocks
    img = np.zeros((h, w, 4))
    img[..., :3] = np.round(rng.uniform(0, 50, size=(h, w, 3)), 1)
    img[..., 3] = 16.0
    img[10:30, 5:60, :3] = 2.5  # runs for the RLE coder
    p = tmp_path / "c.exr"
    p.write_bytes(_exr(img, comp, tiles, half))
    got = accum.read_accum(p)
    want = img.astype(np.float16 if half else np.float32).astype(np.float64)
    np.testing.assert_array_equal(got, want)


def test_bad_files_are_rejected(tmp_path):
    a, _ = _ref_images()
    p = tmp_path / "nocount.exr"
    p.write_bytes(_exr(np.concatenate([a[..., :3], a[..., 3:]], 2), 0, order=("B", "G", "R", "A")))
    with pytest.raises(RtError, match="missing channel count"):
        accum.read_accum(p)
    q = tmp_path / "trunc.exr"
    good = tmp_path / "good.exr"
    accum.write_accum(good, a)
    q.write_bytes(good.read_bytes()[:-40])
    with pytest.raises(RtError):
        accum.read_accum(q)
    big = tmp_path / "big.exr"
    accum.write_accum(big, np.ones((7, 8, 4)))
    with pytest.raises(RtError, match="resolution"):
        accum.merge([good, big])
    with pytest.raises(RtError):
        accum.read_accum(tmp_path / "missing.exr")


def test_rckp_layout(tmp_path):
    rng = np.random.default_rng(3)
    a = rng.uniform(0, 9, size=(5, 7, 4))
    p = tmp_path / "ck.bin"
    accum.write_rckp(p, a, 12)
    b = p.read_bytes()
    assert len(b) == 16 + 5 * 7 * 16
    assert b[:4] == b"RCKP" and struct.unpack("<3I", b[4:16]) == (7, 5, 12)
    np.testing.assert_array_equal(np.frombuffer(b[16:], "<f4").reshape(5, 7, 4), a.astype(np.float32))
