"""RIB ingest (rtcuda.rib): the reference's tokenizer rules
(src/parser/parser.rs and its tests) and SceneBuilder semantics
(src/parser/scene_builder.rs) checked on RIB text written here; the
reference's own fixture files are parsed too when they are available."""
import glob
import math
import os

import numpy as np
import pytest

from rtcuda import abi
from rtcuda.rib import load_rib, load_rib_string, parse_rib


def test_tokenizer_values():
    r = parse_rib('Display "out.ppm" "file" "rgb"\nSphere 1.0 -1.0 1.0 360 # comment\n'
                  'ConcatTransform [1 0 0 0 0 1 0 0 0 0 1 0 -2.5e-1 0 3 1]\n'
                  'Procedural "DelayedReadArchive" ["big.rib"] [-1 1 -1 1 -1 1]\n'
                  'SubdivisionMesh "catmull-clark" [4] [0 1 2 3] [] [] [] [] "P" [0 0 0 1 0 0 1 1 0 0 1 0]')
    assert [n for n, _ in r] == ["Display", "Sphere", "ConcatTransform", "Procedural", "SubdivisionMesh"]
    assert r[0][1] == ["out.ppm", "file", "rgb"]
    assert r[1][1] == [1.0, -1.0, 1.0, 360.0]
    assert len(r[2][1][0]) == 16 and abs(r[2][1][0][12] + 0.25) < 1e-12
    assert r[3][1][1] == ["big.rib"] and r[3][1][2] == [-1.0, 1.0, -1.0, 1.0, -1.0, 1.0]
    assert r[4][1][3] == []


def test_inline_declarations_match_last_word():
    s = load_rib_string('Surface "plastic" "uniform float roughness" [0.25] "Ks" 0.6\nPolygon "P" [0 0 5 1 0 5 0 1 5]')
    m = s.materials[0]
    assert m["specular_ior"] == 1.5 and m["diffuse_gain"] == 0.9 and m["specular_roughness"] == 0.25


CORNELL = """
Format 64 48 1.0
PixelSamples 4 2
Projection "perspective" "fov" [36]
PixelFilter "triangle" 2 2
WorldBegin
  AttributeBegin
    AreaLightSource "arealight" "ceiling" "intensity" [17] "lightcolor" [1 0.9 0.75]
    Translate 0 0 1
    Polygon "P" [-0.25 0.995 3.95  0.25 0.995 3.95  0.25 0.995 4.45  -0.25 0.995 4.45]
  AttributeEnd
  AttributeBegin
    Color 0.73 0.73 0.73
    Surface "matte"
    Polygon "P" [-1 -1 3  1 -1 3  1 -1 5  -1 -1 5]
  AttributeEnd
  AttributeBegin
    Color [0.95 0.93 0.88]
    Surface "metal" "roughness" [0.01]
    Translate 0.4 -0.65 3.9
    Sphere 0.35 -0.35 0.35 360
  AttributeEnd
  LightSource "pointlight" 1 "from" [0 0.5 4] "intensity" [3]
WorldEnd
"""


def test_cornell_like_scene():
    s = load_rib_string(CORNELL)
    assert (s.width, s.height, s.fov, s.spp) == (64, 48, 36.0, 8)
    assert s.filter == abi.FILTER_TRIANGLE and s.filter_width == 2.0
    np.testing.assert_array_equal(s.eye, 0)
    np.testing.assert_array_equal(s.forward, [0, 0, 1])
    np.testing.assert_array_equal(s.right, [1, 0, 0])
    # The area-light quad is a sampleable rect light in world space (after its Translate).
    rect = [l for l in s.lights if l["type"] == abi.LIGHT_RECT]
    assert len(rect) == 1
    np.testing.assert_allclose(rect[0]["p"], (-0.25, 0.995, 4.95))
    np.testing.assert_allclose(rect[0]["e1"], (0.5, 0, 0))
    np.testing.assert_allclose(rect[0]["e2"], (0, 0, 0.5))
    assert rect[0]["intensity"] == 17 and rect[0]["color"] == (1.0, 0.9, 0.75)
    emat = s.materials[0]
    np.testing.assert_allclose(emat["emission"], (17, 15.3, 12.75))
    assert emat["area_light"] == s.lights.index(rect[0])
    # Legacy surfaces map to PbrParams (pbr.rs:104-131); metal roughness floors at 0.02.
    assert s.materials[1]["diffuse_color"] == (0.73, 0.73, 0.73) and s.materials[1]["specular_ior"] == 1.0
    metal = s.materials[2]
    assert metal["diffuse_gain"] == 0.0 and metal["specular_face_color"] == (0.95, 0.93, 0.88)
    assert metal["specular_roughness"] == 0.02
    # Object ids for the id AOV: one per material, from 1.
    assert [m["id"] for m in s.materials] == [1, 2, 3]
    # Point light position as written (no current transform applied).
    pt = [l for l in s.lights if l["type"] == abi.LIGHT_POINT]
    assert pt[0]["p"] == (0.0, 0.5, 4.0) and pt[0]["intensity"] == 3.0
    # The sphere: an analytic quadric of radius 0.35 placed by its Translate.
    kind, params, xf, mat = s.quadrics[0]
    assert kind == abi.QUADRIC_SPHERE and params[:4] == [0.35, -0.35, 0.35, 360.0]
    np.testing.assert_allclose(np.asarray(xf).reshape(3, 4)[:, 3], (0.4, -0.65, 3.9))


def test_transform_order_and_rib_matrices():
    s = load_rib_string("Translate 1 2 3\nRotate 90 0 1 0\nScale 2 3 4\nPolygon \"P\" [0 0 0 1 0 0 0 1 0]\n"
                        "Identity\nConcatTransform [1 0 0 0 0 1 0 0 0 0 1 0 5 6 7 1]\nPolygon \"P\" [0 0 0 1 0 0 0 1 0]")
    xf = s.instance_array()["xf"].reshape(-1, 3, 4)
    r = np.array([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], dtype=np.float64)
    want = np.zeros((3, 4))
    want[:, :3] = r @ np.diag([2, 3, 4])
    want[:, 3] = (1, 2, 3)
    np.testing.assert_allclose(xf[0], want, atol=1e-12)
    np.testing.assert_allclose(xf[1][:, 3], (5, 6, 7))


def test_instancing_and_pxr_lights():
    s = load_rib_string("""
ObjectBegin "tri"
  Translate 0 0 1
  PointsPolygons [3] [0 1 2] "P" [0 0 0 1 0 0 0 1 0]
ObjectEnd
Translate 10 0 0
ObjectInstance "tri"
Translate 0 5 0
ObjectInstance "tri"
AttributeBegin
  Translate 0 3 0
  Scale 2 4 1
  Light "PxrRectLight" "rect" "intensity" [2] "exposure" [1] "lightColor" [1 0.5 0.25]
AttributeEnd
Light "PxrDistantLight" "sun" "intensity" [3] "angleExtent" [1.0]
AttributeBegin
  Scale 3 3 3
  Light "PxrSphereLight" "ball" "intensity" [1]
AttributeEnd
""")
    inst = s.instance_array()
    tri = inst[inst["mesh"] == 0]
    assert len(tri) == 2
    np.testing.assert_allclose(tri["xf"].reshape(-1, 3, 4)[:, :, 3], [(10, 0, 1), (10, 5, 1)])
    rect = s.lights[0]
    assert rect["type"] == abi.LIGHT_RECT and rect["intensity"] == 4.0 and rect["color"] == (1.0, 0.5, 0.25)
    np.testing.assert_allclose(rect["p"], (9, 6, 0))  # the CTM also holds the two Translates above
    np.testing.assert_allclose(rect["e1"], (2, 0, 0))
    np.testing.assert_allclose(rect["e2"], (0, 4, 0))
    sun = s.lights[1]
    assert sun["type"] == abi.LIGHT_DISTANT
    np.testing.assert_allclose(sun["e1"], (0, 0, -1))
    assert abs(sun["radius"] - math.radians(0.5)) < 1e-15
    ball = s.lights[2]
    assert ball["type"] == abi.LIGHT_SPHERE and abs(ball["radius"] - 1.5) < 1e-12
    # Emitters of the area lights are linked to their lights for MIS.
    assert sorted(m["area_light"] for m in s.materials if m["area_light"] >= 0) == [0, 2]


def test_pxr_surface_and_identifiers():
    s = load_rib_string("""
Attribute "identifier" "name" ["teapot"]
Bxdf "PxrSurface" "m" "color diffuseColor" [0.2 0.3 0.4] "float specularRoughness" [0.0]
  "float glassRefractionGain" [1] "float glowGain" [2] "color glowColor" [1 0 0.5] "float presence" [0.5]
Polygon "P" [0 0 0 1 0 0 0 1 0]
Polygon "P" [0 0 1 1 0 1 0 1 1]
Option "background" "color" [0.1 0.2 0.3]
""")
    a, b = s.materials
    assert a["diffuse_color"] == (0.2, 0.3, 0.4) and a["specular_roughness"] == 0.005
    assert a["glass_gain"] == 1.0 and a["glow"] == (2.0, 0.0, 1.0) and a["presence"] == 0.5
    assert a["id"] == b["id"] == 1
    assert s.background == (0.1, 0.2, 0.3)


def test_quadric_requests_are_analytic():
    """Each quadric request becomes an analytic quadric with the request's
    arguments, the current transform and the plain state material
    (scene_builder.rs:813-909); inside an object definition it is skipped."""
    s = load_rib_string('Translate 0 0 5\nSphere 1 -0.5 0.8 270\nCylinder 0.5 -1 1 360\nCone 2 0.5 360\n'
                        'Disk 0.3 1 180\nTorus 1 0.25 0 360 360\nParaboloid 1 0.1 2 360\n'
                        'Hyperboloid 1 0 -1  0.5 0.5 1  360\n'
                        'ObjectBegin 1\nSphere 1 -1 1 360\nObjectEnd\n')
    kinds = [q[0] for q in s.quadrics]
    assert kinds == [abi.QUADRIC_SPHERE, abi.QUADRIC_CYLINDER, abi.QUADRIC_CONE, abi.QUADRIC_DISK,
                     abi.QUADRIC_TORUS, abi.QUADRIC_PARABOLOID, abi.QUADRIC_HYPERBOLOID]
    assert s.quadrics[4][1][:5] == [1.0, 0.25, 0.0, 360.0, 360.0]
    assert s.quadrics[6][1][:7] == [1.0, 0.0, -1.0, 0.5, 0.5, 1.0, 360.0]
    for q in s.quadrics:
        np.testing.assert_allclose(np.asarray(q[2]).reshape(3, 4)[:, 3], (0, 0, 5))
        assert s.materials[q[3]]["emission"] == (0.0, 0.0, 0.0)
    assert any("ObjectBegin" in w for w in s.warnings)


def test_archives_and_missing_files(tmp_path):
    (tmp_path / "part.rib").write_text('Polygon "P" [0 0 0 1 0 0 0 1 0]\n')
    (tmp_path / "main.rib").write_text('ArchiveBegin "inline"\nPolygon "P" [0 0 1 1 0 1 0 1 1]\nArchiveEnd\n'
                                       'ReadArchive "part.rib"\nReadArchive "inline"\nReadArchive "nope.rib"\n')
    s = load_rib(str(tmp_path / "main.rib"))
    assert len(s.meshes) == 2
    assert any("nope.rib" in w for w in s.warnings)


FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fixtures")


def test_reference_fixtures_load():
    files = sorted(glob.glob(os.path.join(FIXTURES, "*.rib")))
    assert files
    for f in files:
        s = load_rib(f)
        assert s.width > 0 and s.height > 0, f
    c = load_rib(os.path.join(FIXTURES, "cornell.rib"))
    assert (c.width, c.height, c.spp) == (600, 600, 64)
    assert [l["type"] for l in c.lights] == [abi.LIGHT_RECT]


def test_rib_presence_binding_and_delayed_archive():
    """A Bxdf "reference float presence" connection becomes a presence
    binding (pattern-driven cutouts), and Procedural "DelayedReadArchive"
    reads its archive at once (scene_builder.rs:384-399)."""
    s = load_rib_string("""
        ArchiveBegin "leaf"
            PointsPolygons [4] [0 1 2 3] "P" [-1 -1 3  1 -1 3  1 1 3  -1 1 3] "st" [0 0 1 0 1 1 0 1]
        ArchiveEnd
        WorldBegin
            Pattern "PxrChecker" "chk" "colorA" [1 1 1] "colorB" [0 0 0]
            Bxdf "PxrSurface" "leafy" "diffuseColor" [0.2 0.6 0.2] "reference float presence" ["chk:resultR"]
            Procedural "DelayedReadArchive" ["leaf"] [-1 1 -1 1 2 4]
        WorldEnd
    """)
    assert s.n_instances == 1
    assert [(f, n) for _, f, n in s.bindings] == [(abi.FIELD_PRESENCE, 0)]
    assert not any("presence" in w for w in s.warnings)


def test_pan_fixture_motion_blocks():
    """The reference's motion-blur demo (pan.rib): transform blocks on three
    placed objects, a deforming PointsPolygons block, thin-lens depth of
    field; the quadric glow spheres in motion blocks stay put, as the
    reference's legacy objects do."""
    s = load_rib(os.path.join(FIXTURES, "pan.rib"))
    assert s.has_motion
    assert len(s.instance_motion) == 3 and len(s.mesh_motion) == 1
    assert s.camera_motion_inv is None
    assert abs(s.lens_radius - 1.0 / 3.2) < 1e-12 and s.focal_distance == 9.0
    assert not any("MotionBegin" in w for w in s.warnings)


# ---- binary RIB (src/parser/binary.rs) -------------------------------------------------------
def _bin_str(t):
    b = t.encode()
    return (bytes([0x90 + len(b)]) if len(b) < 16 else bytes([0xA0, len(b)])) + b


def _encode_binary(reqs):
    """A binary RIB encoder written from RISpec 3.2 Appendix C.2: one request
    definition (0314) per name, then uses (0246); numbers as 32-bit floats
    (0244) or small integers (0200); strings length-prefixed; arrays kept as
    ASCII brackets."""
    import struct
    out, codes = bytearray(), {}
    for name, vals in reqs:
        if name not in codes:
            codes[name] = len(codes)
            out += bytes([0xCC, codes[name]]) + _bin_str(name)
        out += bytes([0xA6, codes[name]])
        for v in vals:
            items = v if isinstance(v, list) else [v]
            if isinstance(v, list):
                out += b"["
            for x in items:
                if isinstance(x, str):
                    out += _bin_str(x)
                elif float(x).is_integer() and -128 <= x < 128:
                    out += bytes([0x80]) + struct.pack(">b", int(x))
                else:
                    out += bytes([0xA4]) + struct.pack(">f", x)
            if isinstance(v, list):
                out += b"]"
    return bytes(out)


def test_binary_rib_loads_like_text(tmp_path):
    from rtcuda.rib import looks_binary
    text = CORNELL.replace("0.995", "0.5").replace("0.73", "0.75").replace("0.65", "0.625")
    data = _encode_binary(parse_rib(text))
    assert looks_binary(data) and not looks_binary(text.encode())
    (tmp_path / "b.rib").write_bytes(data)
    (tmp_path / "t.rib").write_text(text)
    a, b = load_rib(str(tmp_path / "t.rib")), load_rib(str(tmp_path / "b.rib"))
    assert (a.width, a.height, a.fov, a.spp) == (b.width, b.height, b.fov, b.spp)
    assert a.materials == b.materials and a.lights == b.lights
    for (pa, ia, na), (pb, ib, nb) in zip(a.meshes, b.meshes):
        np.testing.assert_array_equal(pa, pb)
        np.testing.assert_array_equal(ia, ib)
    np.testing.assert_array_equal(a.instance_array(), b.instance_array())


def test_binary_codes_tokens_fixed_point_double():
    import struct
    from rtcuda.rib import decode_binary
    data = (bytes([0xCC, 7]) + _bin_str("Translate")
            + bytes([0xC8, 5]) + _bin_str("roughness")                          # string token 5
            + bytes([0xA6, 7]) + bytes([0x85]) + struct.pack(">h", 384)         # fixed point: 384
            + bytes([0x89]) + struct.pack(">i", -640)[1:]                       # 2 int + 1 fraction bytes: -2.5
            + bytes([0xA5]) + struct.pack(">d", 0.1)                            # double
            + b"\n# comment \xff stays\n"
            + bytes([0xCD, 5]))                                                 # token reference
    r = parse_rib(decode_binary(data))
    assert r[0] == ("Translate", [384.0, -2.5, 0.1, "roughness"])


def test_binary_decoder_is_total_on_noise():
    from rtcuda.rib import RibError, decode_binary
    rng = np.random.default_rng(0x9E3779B9)
    for _ in range(300):
        data = bytes(rng.integers(0, 256, size=int(rng.integers(0, 200)), dtype=np.uint8))
        try:
            decode_binary(data)
        except RibError:
            pass


def test_pxr_dome_light():
    s = load_rib_string('Light "PxrDomeLight" "sky" "intensity" [2] "exposure" [1] "lightColor" [0.5 0.5 1]\n'
                        'Light "PxrDomeLight" "env" "string lightColorMap" ["sky.exr"]')
    assert [l["type"] for l in s.lights] == [abi.LIGHT_DOME, abi.LIGHT_DOME]
    assert s.lights[0]["intensity"] == 4.0 and s.lights[0]["color"] == (0.5, 0.5, 1.0)
    assert any("sky.exr" in w for w in s.warnings) and s.env is None  # a map that cannot be read: constant dome


def test_pxr_dome_light_reads_hdr_map(tmp_path):
    from test_envmap_cpu import _encode, _rgbe
    img = np.full((4, 16, 3), 0.5, np.float32)
    (tmp_path / "sky.hdr").write_bytes(_encode(_rgbe(img)))
    (tmp_path / "s.rib").write_text('Light "PxrDomeLight" "sky" "string lightColorMap" ["sky.hdr"]\n')
    s = load_rib(str(tmp_path / "s.rib"))
    assert s.env is not None and s.env[0] == 0 and s.env[1].shape == (4, 16, 3)
    np.testing.assert_allclose(s.env[1], 0.5, atol=1 / 256)  # RGBE has 8-bit mantissas


def test_pattern_graph_binds_to_bxdf():
    """scene_builder.rs:1993-2023: two Pattern nodes, one Bxdf connection;
    the checker cell (0, 0) is red, mixed 25% toward green."""
    import oracle
    s = load_rib_string('''
        Format 64 64 1.0
        WorldBegin
            Pattern "PxrChecker" "check" "colorA" [1 0 0] "colorB" [0 0 1] "sScale" [4] "tScale" [4]
            Pattern "PxrMix" "blend" "reference color color1" ["check:resultRGB"] "color2" [0 1 0] "mix" [0.25]
            Bxdf "PxrSurface" "mat" "reference color diffuseColor" ["blend:resultRGB"] "specularIor" [1]
            Sphere 1 -1 1 360
        WorldEnd''')
    assert len(s.patterns) == 2
    assert s.bindings == [(len(s.materials) - 1, abi.PATTERN_FIELDS["diffuseColor"], 1)]
    c = oracle.pattern_eval(s, 1, [[0.1, 0.1, 0.0, 0.0, 0.0, 0.0]])[0]
    assert abs(c[0] - 0.75) < 1e-9 and abs(c[1] - 0.25) < 1e-9


def test_pattern_requests_and_connections():
    s = load_rib_string('''
        Pattern "PxrFractal" "n" "frequency" [2] "layers" [3] "gain" [0.4]
        Pattern "PxrColorCorrect" "cc" "reference color inputRGB" ["n:resultRGB"] "gamma" [2] "saturation" [0.5]
        Pattern "PxrRamp" "r" "positions" [0 0.5 1] "colors" [0 0 0  1 0 0  1 1 1] "axis" "t"
        Pattern "PxrTexture" "tex" "filename" "wood.tex"
        Pattern "PxrChecker" "nohandle_is_fine" 
        Bxdf "PxrSurface" "m" "reference color diffuseColor" ["cc:resultRGB"] "reference float presence" ["n:resultF"]
          "reference color specularFaceColor" ["tex:resultRGB"] "reference float bogus" ["n:resultF"]
        Polygon "P" [0 0 1  1 0 1  1 1 1]''')
    kinds = [n["type"] for n in s.patterns]
    assert kinds == [abi.PATTERN_FRACTAL, abi.PATTERN_COLOR_CORRECT, abi.PATTERN_RAMP, abi.PATTERN_TEXTURE,
                     abi.PATTERN_CHECKER]
    assert s.patterns[0]["octaves"] == 3 and s.patterns[0]["gain"] == 0.4
    assert s.patterns[1]["inputs"] == (0,) and s.patterns[1]["gamma"] == 2.0
    assert s.patterns[2]["use_t"] and list(s.patterns[2]["ramp"][0]) == [0.0, 0.5, 1.0]
    assert s.patterns[3]["texture"] == -1  # wood.tex cannot be read: magenta
    assert s.patterns[4]["scale"] == (8.0, 8.0) and s.patterns[4]["color_a"] == (1.0, 1.0, 1.0)
    assert [b[1:] for b in s.bindings] == [(abi.PATTERN_FIELDS["diffuseColor"], 1),
                                           (abi.PATTERN_FIELDS["presence"], 0),
                                           (abi.PATTERN_FIELDS["specularFaceColor"], 3)]
    w = " | ".join(s.warnings)
    assert "wood.tex" in w and "bogus" in w


def test_st_primvar():
    s = load_rib_string('PointsPolygons [4] [0 1 2 3] "P" [0 0 1  1 0 1  1 1 1  0 1 1] "st" [0 0  1 0  1 1  0 1]\n'
                        'PointsPolygons [3] [0 1 2] "P" [0 0 1  1 0 1  1 1 1] "st" [0 0  1 0]\n')
    # Wrong-length st is ignored.
    assert sorted(s.mesh_st) == [0]
    np.testing.assert_array_equal(s.mesh_st[0], [[0, 0], [1, 0], [1, 1], [0, 1]])


def test_media_requests_and_subsurface():
    """Interior / Atmosphere (scene_builder.rs:324-373) and the PxrSurface
    subsurface parameters (pbr.rs:174-183)."""
    s = load_rib_string("""
Format 8 8 1
Atmosphere "haze" "sigma_a" [0.1 0.2 0.3] "sigma_s" [0.5 0.5 0.5] "g" [0.3]
WorldBegin
  AttributeBegin
    Interior "cloud" "sigma_s" [4 4 4] "density" ["fbm"] "frequency" [0.2] "octaves" [3] "coverage" [0.7]
    Bxdf "PxrSurface" "hull" "diffuseGain" [0] "specularIor" [1]
    Sphere 1 -1 1 360
  AttributeEnd
  Bxdf "PxrSurface" "skin" "subsurfaceGain" [0.8] "subsurfaceColor" [0.9 0.4 0.3] "subsurfaceDmfp" [0.05]
  Polygon "P" [-1 -1 5  1 -1 5  1 1 5  -1 1 5]
WorldEnd
""")
    assert len(s.media) == 2 and s.atmosphere == 0
    haze, cloud = s.media
    assert haze["sigma_a"] == (0.1, 0.2, 0.3) and haze["g"] == 0.3 and haze["max_distance"] == 1200.0
    assert haze["density"] == abi.DENSITY_NONE
    assert cloud["density"] == abi.DENSITY_FBM and cloud["octaves"] == 3 and cloud["frequency"] == 0.2
    assert cloud["coverage"] == 0.7 and cloud["gain"] == 0.55 and cloud["max_distance"] == float("inf")
    assert cloud["sigma_a"] == (0.1, 0.1, 0.1)  # the request's defaults
    hull = s.materials[s.quadrics[0][3]]
    assert hull["interior"] == 1 and hull["diffuse_gain"] == 0.0
    skin = s.materials[-1]
    assert skin["interior"] == -1  # AttributeEnd restored the state
    assert skin["subsurface_gain"] == 0.8 and skin["subsurface_dmfp"] == (0.05, 0.05, 0.05)
    assert skin["subsurface_color"] == (0.9, 0.4, 0.3)


def test_clouds_fixture_media():
    s = load_rib(os.path.join(FIXTURES, "clouds.rib"))
    assert len(s.media) == 3 and s.atmosphere == 0
    assert [m["density"] for m in s.media] == [abi.DENSITY_NONE, abi.DENSITY_FBM, abi.DENSITY_FBM]
    assert s.media[0]["max_distance"] == 900.0
    hulls = [q for q in s.quadrics if s.materials[q[3]]["interior"] >= 0]
    assert len(hulls) == 9

