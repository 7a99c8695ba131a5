"""The C ABI library without a GPU: it loads, exports every function the
headers declare, and rejects invalid scenes on the host before touching CUDA."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from rtcuda import abi, backend, scene, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("rt_cuda.h", "rt_guide.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(rt_[a-z_0-9]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = backend.lib()
    declared = declared_functions()
    assert declared, "no declarations parsed"
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    from rtcuda import guide
    assert declared == set(backend.EXPORTS) | set(guide.EXPORTS)


def test_descriptor_layouts_match_headers():
    sizes = {"rt_mesh_desc": 40, "rt_instance_desc": 104, "rt_material_desc": 376, "rt_light_desc": 120,
             "rt_camera_desc": 160, "rt_params": 72, "rt_pattern_desc": 264, "rt_pattern_binding": 16,
             "rt_texture_desc": 16, "rt_ies_desc": 112, "rt_quadric_desc": 168, "rt_scene_desc": 392, "rt_medium_desc": 136,
             "rt_curves_desc": 40, "rt_instance_motion": 104, "rt_mesh_motion": 16}
    text = open(os.path.join(ROOT, "include", "rt_scene.h")).read()
    for name, size in sizes.items():
        assert f"sizeof({name}) == {size}" in text
    assert C.sizeof(abi.RtMaterialDesc) == 376 and C.sizeof(abi.RtSceneDesc) > 0


def _create(s, **kw):
    h = C.c_void_p()
    d = s.desc()
    p = abi.make_params(**kw)
    rc = backend.lib().rt_session_create(C.byref(d), C.byref(p), C.byref(h))
    return rc, backend.lib().rt_last_error().decode()


def test_bad_index_rejected_on_host():
    s = scene.Scene(4, 4)
    s.meshes.append((np.zeros((3, 3), np.float32), np.array([[0, 1, 7]], np.uint32), None))
    s.add_instance(0, s.add_material(scene.matte((0.5, 0.5, 0.5))))
    rc, msg = _create(s, bvh_build="host")  # the device builder validates on the GPU
    assert rc == -1 and "index out of range" in msg


def test_missing_material_rejected_on_host():
    s = scene.Scene(4, 4)
    s.add_instance(s.add_mesh([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 2]]), 3)
    rc, msg = _create(s)
    assert rc == -1 and "missing mesh or material" in msg


def test_non_finite_vertex_rejected_on_host():
    s = scene.Scene(4, 4)
    s.add_instance(s.add_mesh([[0, 0, np.nan], [1, 0, 0], [0, 1, 0]], [[0, 1, 2]]),
                   s.add_material(scene.matte((0.5, 0.5, 0.5))))
    rc, msg = _create(s, bvh_build="host")
    assert rc == -1 and "non-finite" in msg


def test_bad_max_depth_rejected():
    rc, msg = _create(scenes.cornell_box(4, 4), max_depth=0)
    assert rc == -1 and "max_depth" in msg


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(backend, "_lib", None)
    monkeypatch.setattr(backend, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(backend.RtError):
        backend.lib()
