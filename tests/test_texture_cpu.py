"""File textures on the CPU: the .tex writer/reader against the reference's
tex.rs tests (src/texture/tex.rs:253-311), the oracle's texture lookups
against its cache tests (src/texture/cache.rs:393-477), the mip chain the
CUDA backend builds against the writer's, PNG decoding, and PxrTexture /
triplanar requests read from RIB."""
import struct
import zlib

import numpy as np

import oracle
from rtcuda import abi, scene, textures
from rtcuda.rib import load_rib_string


def checker(w, h):
    x, y = np.arange(w)[None, :], np.arange(h)[:, None]
    v = np.where((x // 8 + y // 8) % 2 == 0, 1.0, 0.25).astype(np.float32)
    return np.stack([v, v * np.float32(0.5), np.full_like(v, 0.1)], -1)


def gradient(w, h):
    x, y = np.arange(w)[None, :] / (w - 1), np.arange(h)[:, None] / (h - 1)
    return np.stack(np.broadcast_arrays(x, y, 0.5), -1).astype(np.float32)


def test_tex_round_trip_and_mips(tmp_path):
    img = checker(70, 50)
    path = tmp_path / "a.tex"
    textures.write_tex(path, img)
    data = path.read_bytes()
    w, h, mips = textures.read_tex_header(data)
    assert (w, h) == (70, 50)
    assert [m[:2] for m in mips] == [(70, 50), (35, 25), (17, 12), (8, 6), (4, 3), (2, 1), (1, 1)]
    assert mips[0][2:4] == (3, 2)
    assert textures.read_tex_tile(data, 0, 1, 0)[20, 40 - 32, 0] == img[20, 40, 0]
    top = textures.read_tex_tile(data, len(mips) - 1, 0, 0)[0, 0, 0]
    assert 0.25 < top < 1.0
    np.testing.assert_array_equal(textures.read_tex(path), img)


def test_broken_tex_files_raise(tmp_path):
    textures.write_tex(tmp_path / "ok.tex", checker(40, 40))
    data = (tmp_path / "ok.tex").read_bytes()
    for k, broken in enumerate((data[:20], data[:40], data[:300], b"XTEX" + data[4:])):
        (tmp_path / f"b{k}.tex").write_bytes(broken)
        try:
            textures.read_tex(tmp_path / f"b{k}.tex")
            raise AssertionError(f"broken file {k} read")
        except textures.TextureError:
            pass


def test_edge_tiles_replicate(tmp_path):
    img = checker(40, 40)
    path = tmp_path / "e.tex"
    textures.write_tex(path, img)
    assert textures.read_tex_tile(path.read_bytes(), 0, 1, 1)[20, 20, 0] == img[39, 39, 0]


def test_sample_center_and_wrap():
    img = gradient(128, 128)
    c = oracle.texture_sample(img, [[0.5, 0.5, 0.0]])[0]
    assert abs(c[0] - 0.5) < 0.02 and abs(c[1] - 0.5) < 0.02
    assert oracle.texture_sample(img, [[1.02, 0.5, 0.0]])[0][0] < 0.1
    assert np.all(oracle.texture_sample(img, [[1.5, 0.5, 0.0]], wrap=abi.WRAP_BLACK)[0] == 0.0)
    top = oracle.texture_sample(img, [[0.25, 0.75, 10.0]])[0]
    assert abs(top[0] - 0.5) < 0.05 and abs(top[2] - 0.5) < 0.01


def test_ewa_preserves_detail_across_anisotropy():
    x = np.arange(256)
    v = np.where((x // 8) % 2 == 0, 1.0, 0.0).astype(np.float32)
    img = np.repeat(np.repeat(v[None, :, None], 256, 0), 3, 2)
    du, dv = (0.0, 64.0 / 256.0), (1.0 / 256.0, 0.0)
    on, off = oracle.texture_sample(img, [[4.5 / 256, 0.5, *du, *dv], [12.5 / 256, 0.5, *du, *dv]], ewa=True)
    assert abs(on[0] - off[0]) > 0.5
    on_t, off_t = oracle.texture_sample(img, [[4.5 / 256, 0.5, 64.0 / 256], [12.5 / 256, 0.5, 64.0 / 256]])
    assert abs(on_t[0] - off_t[0]) < 0.2


def test_oracle_mip_chain_matches_the_tex_writer():
    img = checker(70, 50) * np.float32(0.7) + gradient(70, 50) * np.float32(0.3)
    chain = textures.mip_chain(img)
    for level in (1, 3):
        m = chain[level]
        h, w = m.shape[:2]
        base = 70.0
        ys, xs = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
        q = np.stack([(xs.ravel() + 0.5) / w, (ys.ravel() + 0.5) / h, np.full(xs.size, 2.0 ** level / base)], -1)
        got = oracle.texture_sample(img, q, wrap=abi.WRAP_CLAMP)
        np.testing.assert_allclose(got, m.reshape(-1, 3), rtol=0, atol=2e-7)
    last = oracle.texture_sample(img, [[0.3, 0.6, 1e3]])[0]  # four bilinear taps of the 1x1 level
    np.testing.assert_allclose(last, chain[-1][0, 0], rtol=0, atol=2e-7)


def _filter_row(line, prev, ftype, bpp=3):
    """The encoder side of PNG filter `ftype` for one row (ints 0-255)."""
    out = []
    for i, x in enumerate(line):
        a = line[i - bpp] if i >= bpp else 0
        b = prev[i]
        c = prev[i - bpp] if i >= bpp else 0
        if ftype == 0:
            p = 0
        elif ftype == 1:
            p = a
        elif ftype == 2:
            p = b
        elif ftype == 3:
            p = (a + b) >> 1
        else:
            pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
            p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
        out.append((x - p) & 0xFF)
    return bytes(out)


def _png(a, ftype=0):
    h, w, _ = a.shape
    rows, prev = [], [0] * (w * 3)
    for y in range(h):
        line = [int(v) for v in a[y].reshape(-1)]
        f = ftype if ftype >= 0 else y % 5  # -1: a different filter on every row
        rows.append(bytes([f]) + _filter_row(line, prev, f))
        prev = line

    def chunk(k, b):
        return struct.pack(">I", len(b)) + k + b + struct.pack(">I", zlib.crc32(k + b) & 0xFFFFFFFF)
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(b"".join(rows))) + chunk(b"IEND", b""))


def test_png_decode_and_srgb():
    a = np.random.default_rng(3).integers(0, 256, (6, 9, 3)).astype(np.uint8)
    for ftype in (0, 1, 2, 3, 4, -1):
        np.testing.assert_allclose(textures.decode_png(_png(a, ftype)), a / 255.0, atol=1e-7)
    full = _png(a, 4)
    for broken in (full[:60] + full[-12:], full[:40], full[:20], b"not a png"):
        try:
            textures.decode_png(broken)
            raise AssertionError("a broken PNG decoded")
        except textures.TextureError:
            pass
    lin = textures.srgb_to_linear(np.array([0.0, 0.04045, 0.5, 1.0], np.float32))
    np.testing.assert_allclose(lin, [0.0, 0.04045 / 12.92, ((0.5 + 0.055) / 1.055) ** 2.4, 1.0], rtol=1e-6)


def test_rib_texture_nodes(tmp_path):
    textures.write_tex(tmp_path / "wood.tex", checker(16, 16))
    (tmp_path / "paint.png").write_bytes(_png(np.full((2, 2, 3), 255, np.uint8)))
    s = load_rib_string('''
        Pattern "PxrTexture" "wood" "string filename" ["wood.tex"] "string wrapMode" ["clamp"] "scaleS" [2]
        Pattern "triplanar" "tri" "string filename" ["paint.png"] "frequency" [3]
        Pattern "PxrTexture" "gone" "string filename" ["missing.tex"]
        Bxdf "PxrSurface" "m" "reference color diffuseColor" ["wood:resultRGB"]
        Polygon "P" [0 0 1  1 0 1  1 1 1]''', base_dir=str(tmp_path))
    wood, tri, gone = s.patterns
    assert wood["type"] == abi.PATTERN_TEXTURE and wood["wrap"] == abi.WRAP_CLAMP and wood["scale"] == (2.0, 1.0)
    assert tri["type"] == abi.PATTERN_TRIPLANAR and tri["frequency"] == 3.0
    assert gone["texture"] == -1 and any("missing.tex" in w for w in s.warnings)
    assert len(s.textures) == 2
    np.testing.assert_array_equal(s.textures[wood["texture"]], checker(16, 16))
    np.testing.assert_allclose(s.textures[tri["texture"]], 1.0)
    # Missing texture: magenta; a texture node reads t up (row 0 at t = 1).
    c = oracle.pattern_eval(s, 2, [[0.5, 0.5, 0, 0, 0, 0]])[0]
    np.testing.assert_array_equal(c, [1.0, 0.0, 1.0])
    top_left = oracle.pattern_eval(s, 0, [[0.01, 0.99, 0, 0, 0, 0]])[0]
    np.testing.assert_allclose(top_left, checker(16, 16)[0, 0], atol=1e-6)


def test_texture_pattern_on_a_quad_in_the_oracle():
    s = scene.Scene(4, 4)
    t = s.add_texture(checker(32, 32))
    n = s.add_texture_node(t, scale=(1.0, 1.0))
    m = s.add_material(scene.matte((1, 1, 1)))
    s.bind_pattern(m, "diffuseColor", n)
    q = s.add_mesh([[0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], [[0, 1, 2], [0, 2, 3]],
                   st=[[0, 0], [1, 0], [1, 1], [0, 1]])
    s.add_instance(q, m)
    ctx = [[0.2, 0.8, 0.2, 0.8, 1.0, 0, 0, -1, 0.0, 0, 0, 0, 0]]
    np.testing.assert_allclose(oracle.pattern_eval(s, n, ctx)[0], checker(32, 32)[6, 6], atol=1e-6)


def _udim_scene():
    """Four constant-colour tiles 1001, 1002, 1011, 1012 as one UDIM set."""
    s = scene.Scene(4, 4)
    colors = {1001: (1.0, 0.0, 0.0), 1002: (0.0, 1.0, 0.0), 1011: (0.0, 0.0, 1.0), 1012: (1.0, 1.0, 0.0)}
    tiles = {t: s.add_texture(np.tile(np.array(c, np.float32), (4, 4, 1))) for t, c in colors.items()}
    return s, s.add_texture_node(-1, udim=tiles), colors


def test_udim_tile_pick():
    """pattern.rs:350-373: (0.5, 0.5) is tile 1001, (1.3, 1.4) tile 1012,
    (5.0, 0.0) a tile outside the set (magenta)."""
    s, node, colors = _udim_scene()
    c = oracle.pattern_eval(s, node, [[0.5, 0.5, 0, 0, 0, 0], [1.3, 1.4, 0, 0, 0, 0], [5.0, 0.0, 0, 0, 0, 0],
                                      [1.5, 0.2, 0, 0, 0, 0], [0.2, 1.5, 0, 0, 0, 0]])
    np.testing.assert_allclose(c, [colors[1001], colors[1012], (1, 0, 1), colors[1002], colors[1011]], atol=1e-6)


def test_rib_udim_files(tmp_path):
    for tile, v in ((1001, 0.25), (1012, 0.75)):
        textures.write_tex(tmp_path / f"paint.{tile}.tex", np.full((2, 2, 3), v, np.float32))
    s = load_rib_string('Pattern "PxrTexture" "p" "string filename" ["paint.<UDIM>.tex"]\n'
                        'Pattern "PxrTexture" "q" "string filename" ["none.<UDIM>.tex"]', base_dir=str(tmp_path))
    assert sorted(s.patterns[0]["udim"]) == [1001, 1012]
    assert s.patterns[1]["texture"] == -1 and "udim" not in s.patterns[1]
    assert any("no UDIM tiles" in w for w in s.warnings)
    c = oracle.pattern_eval(s, 0, [[0.5, 0.5, 0, 0, 0, 0], [1.5, 1.5, 0, 0, 0, 0]])
    np.testing.assert_allclose(c[:, 0], [0.25, 0.75], atol=1e-6)
