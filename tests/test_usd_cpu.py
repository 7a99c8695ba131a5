"""USD (.usda) ingest on the CPU: the reference's own stage test
(src/parser/usd.rs:840-936) and the translation rules of usd.rs (xform
ops, UsdPreviewSurface, lights, Mesh / Sphere / Cube, the camera chain,
Z-up stages), checked through the scene the RIB builder makes."""
import math

import numpy as np

from rtcuda import abi
from rtcuda.rib import load_rib_string
from rtcuda.usd import load_usda_string, usda_to_requests

STAGE = '''#usda 1.0
(
    defaultPrim = "World"
    upAxis = "Y"
)

def Xform "World"
{
    def Camera "Cam"
    {
        float focalLength = 35
        float horizontalAperture = 36
        double3 xformOp:translate = (0, 1, 10)
        uniform token[] xformOpOrder = ["xformOp:translate"]
    }

    def DistantLight "Sun"
    {
        float inputs:intensity = 2.5
        color3f inputs:color = (1, 0.9, 0.8)
    }

    def Scope "Materials"
    {
        def Material "Red"
        {
            token outputs:surface.connect = </World/Materials/Red/PBR.outputs:surface>
            def Shader "PBR"
            {
                uniform token info:id = "UsdPreviewSurface"
                color3f inputs:diffuseColor = (0.8, 0.1, 0.05)
                float inputs:roughness = 0.35
                float inputs:metallic = 0
            }
        }
    }

    def Xform "Geo"
    {
        double3 xformOp:translate = (0, 0, 0)
        uniform token[] xformOpOrder = ["xformOp:translate"]

        def Mesh "Quad"
        {
            int[] faceVertexCounts = [4]
            int[] faceVertexIndices = [0, 1, 2, 3]
            point3f[] points = [(-5, 0, -5), (5, 0, -5), (5, 0, 5), (-5, 0, 5)]
            rel material:binding = </World/Materials/Red>
        }

        def Sphere "Ball"
        {
            double radius = 1.5
            double3 xformOp:translate = (0, 1.5, 0)
            uniform token[] xformOpOrder = ["xformOp:translate"]
        }
    }
}
'''


def _xf(s, k):
    inst = s.instance_array()
    m = np.eye(4)
    m[:3, :] = inst["xf"][k].reshape(3, 4)
    return m


def test_usda_parses_and_builds():
    s = load_usda_string(STAGE)
    assert len(s.lights) == 1 and s.lights[0]["type"] == abi.LIGHT_DISTANT
    assert s.lights[0]["intensity"] == 2.5 and s.lights[0]["color"] == (1.0, 0.9, 0.8)
    inst = s.instance_array()
    assert len(inst) == 2  # the quad and the (tessellated) sphere
    assert abs(s.fov - 54.43) < 0.1
    mat = s.materials[inst["mat"][0]]
    assert abs(mat["diffuse_color"][0] - 0.8) < 1e-6 and abs(mat["specular_roughness"] - 0.35) < 1e-6
    center = _xf(s, 1) @ np.array([0.0, 0.0, 0.0, 1.0])
    assert center[2] > 5.0, center


def test_xform_ops_match_their_rib():
    usda = '''def Xform "A" {
        double3 xformOp:translate = (1, 2, 3)
        float3 xformOp:rotateXYZ = (10, 20, 30)
        float3 xformOp:scale = (2, 1, 0.5)
        uniform token[] xformOpOrder = ["xformOp:translate", "xformOp:rotateXYZ", "xformOp:scale"]
        def Mesh "M" { int[] faceVertexCounts = [3]  int[] faceVertexIndices = [0, 1, 2]
                       point3f[] points = [(0, 0, 0), (1, 0, 0), (0, 1, 0)] }
    }'''
    s = load_usda_string(usda)
    rib = load_rib_string('Projection "perspective" "fov" [45]\nScale 1 1 -1\nWorldBegin\nTranslate 1 2 3\n'
                          'Rotate 30 0 0 1\nRotate 20 0 1 0\nRotate 10 1 0 0\nScale 2 1 0.5\n'
                          'PointsPolygons [3] [0 1 2] "P" [0 0 0 1 0 0 0 1 0]\nWorldEnd')
    np.testing.assert_allclose(_xf(s, 0), _xf(rib, 0), atol=1e-12)
    # rotateXYZ rotates points about x first, then y, then z.
    r = _xf(s, 0)[:3, :3] @ np.diag([0.5, 1.0, 2.0])
    rz, ry, rx = (np.radians(a) for a in (30, 20, 10))
    Rx = np.array([[1, 0, 0], [0, math.cos(rx), -math.sin(rx)], [0, math.sin(rx), math.cos(rx)]])
    Ry = np.array([[math.cos(ry), 0, math.sin(ry)], [0, 1, 0], [-math.sin(ry), 0, math.cos(ry)]])
    Rz = np.array([[math.cos(rz), -math.sin(rz), 0], [math.sin(rz), math.cos(rz), 0], [0, 0, 1]])
    np.testing.assert_allclose(np.diag([1, 1, -1]) @ Rz @ Ry @ Rx, r, atol=1e-12)


def test_materials_lights_and_shapes():
    usda = '''#usda 1.0
(
    upAxis = "Z"
)
def Scope "Looks" {
    def Material "Gold" { def Shader "S" { uniform token info:id = "UsdPreviewSurface"
        color3f inputs:diffuseColor = (1, 0.8, 0.3)  float inputs:metallic = 1  float inputs:roughness = 0.01 } }
    def Material "Lamp" { def Shader "S" { uniform token info:id = "UsdPreviewSurface"
        color3f inputs:emissiveColor = (4, 4, 2)  float inputs:opacity = 0.5  float inputs:ior = 1.33 } }
}
def Cube "Box" ( prepend references = @other.usda@ ) { double size = 4  rel material:binding = </Looks/Gold> }
def Mesh "Tri" { int[] faceVertexCounts = [3]  int[] faceVertexIndices = [0, 1, 2]
    point3f[] points = [(0, 0, 0), (1, 0, 0), (0, 1, 0)]  normal3f[] normals = [(0, 0, 1), (0, 0, 1), (0, 0, 1)]
    texCoord2f[] primvars:st = [(0, 0), (1, 0), (0, 1)]  rel material:binding = </Looks/Lamp> }
def SphereLight "Bulb" { float inputs:intensity = 3  float inputs:exposure = 1  float inputs:radius = 0.25
    double3 xformOp:translate = (0, 0, 3) }
def RectLight "Panel" { float inputs:width = 2  float inputs:height = 0.5 }
def DomeLight "Sky" { float inputs:intensity = 0.5 }
'''
    s = load_usda_string(usda)
    inst = s.instance_array()
    gold = s.materials[inst["mat"][0]]
    assert gold["diffuse_gain"] == 0.0 and gold["specular_face_color"] == (1.0, 0.8, 0.3)
    assert gold["specular_roughness"] == 0.02  # roughness floored at 0.02
    lamp = s.materials[inst["mat"][1]]
    assert lamp["glow"] == (4.0, 4.0, 2.0) and lamp["presence"] == 0.5 and lamp["specular_ior"] == 1.33
    assert 0 in s.mesh_st or 1 in s.mesh_st
    assert s.meshes[inst["mesh"][1]][2] is not None  # normals carried
    kinds = [l["type"] for l in s.lights]
    assert abi.LIGHT_SPHERE in kinds and abi.LIGHT_RECT in kinds and abi.LIGHT_DOME in kinds
    sphere = next(l for l in s.lights if l["type"] == abi.LIGHT_SPHERE)
    assert sphere["intensity"] == 6.0  # 3 * 2^1
    assert any("composition metadata" in w for w in s.warnings)
    # The cube spans 4 units; Z-up puts its +z extent on our +y (then the
    # camera flip takes z to -z).
    P = s.meshes[inst["mesh"][0]][0]
    assert np.allclose(np.abs(P), 2.0)
    reqs, _ = usda_to_requests(usda)
    assert ("Rotate", [-90.0, 1.0, 0.0, 0.0]) in reqs[:reqs.index(("WorldBegin", []))]


def test_translation_round_trips_through_rib_text():
    from rtcuda.rib import format_rib, parse_rib
    from rtcuda.usd import usda_to_rib
    reqs, _ = usda_to_requests(STAGE)
    text = usda_to_rib(STAGE)
    back = parse_rib(text)
    assert [r[0] for r in back] == [r[0] for r in reqs]
    for (n0, v0), (n1, v1) in zip(reqs, back):
        flat0 = [x for v in v0 for x in (v if isinstance(v, list) else [v])]
        flat1 = [x for v in v1 for x in (v if isinstance(v, list) else [v])]
        assert len(flat0) == len(flat1), n0
        for a, b in zip(flat0, flat1):
            assert a == b
    # The RIB text builds the same scene as the stage.
    a, b = load_usda_string(STAGE), load_rib_string(text)
    np.testing.assert_array_equal(a.instance_array()["xf"], b.instance_array()["xf"])
    assert a.materials == b.materials and a.fov == b.fov
    assert format_rib([("Attribute", ["identifier", "name", ['say "hi"']])]) == \
        'Attribute "identifier" "name" ["say \\"hi\\""]\n'
