"""IES profiles on the CPU: the parser and the oracle's evaluation against
the reference's own test (src/scene/ies.rs:168-205, its hand-written narrow
downlight), RIB point lights that name a profile, and the host checks the
CUDA backend makes on profiles."""
import ctypes as C

import numpy as np
import pytest

import oracle
from rtcuda import abi, backend, scene
from rtcuda.ies import IesError, parse_ies
from rtcuda.rib import load_rib_string

# The reference test's profile: 5 vertical angles, 1 horizontal angle.
DOWNLIGHT = ("IESNA:LM-63-2002\n[TEST] hand-written narrow downlight\nTILT=NONE\n"
             "1 1000 1 5 1 1 2 0.1 0.1 0.1\n1.0 1.0 100\n0 20 40 60 90\n0\n1000 800 200 20 0\n")


def test_parse_and_evaluate():
    prof = parse_ies(DOWNLIGHT)
    assert len(prof[0]) == 5 and len(prof[1]) == 1
    t30 = np.radians(30.0)
    dirs = [[0, -1, 0], [1, 0, 0], [0, 1, 0], [np.sin(t30), -np.cos(t30), 0]]
    cd, f = oracle.ies_eval(prof, dirs)
    assert abs(cd[0] - 1000.0) < 1e-6 and cd[1] < 1.0 and cd[2] < 1.0
    assert abs(cd[3] - 500.0) < 1.0
    assert f[0] > 2.0


def test_parse_errors_and_multiplier():
    with pytest.raises(IesError, match="TILT"):
        parse_ies("no tilt here")
    with pytest.raises(IesError, match="TILT=NONE"):
        parse_ies("TILT=INCLUDE\n1 2 3")
    with pytest.raises(IesError, match="truncated"):
        parse_ies("TILT=NONE\n1 1000 1 5")
    doubled = parse_ies(DOWNLIGHT.replace("1 1000 1 5", "1 1000 2 5"))
    np.testing.assert_array_equal(doubled[2], parse_ies(DOWNLIGHT)[2] * 2)


def test_symmetry_folding():
    # Quadrant-symmetric (last horizontal angle 90): phi folds into [0, 90].
    v = np.array([0.0, 90.0, 180.0])
    h = np.array([0.0, 90.0])
    c = np.array([[10.0, 10.0, 10.0], [30.0, 30.0, 30.0]])
    d = [[1, 0, 0], [0, 0, 1], [-1, 0, 0], [0, 0, -1], [np.cos(np.radians(135)), 0, np.sin(np.radians(135))]]
    cd, _ = oracle.ies_eval((v, h, c), d)
    np.testing.assert_allclose(cd, [10, 30, 10, 30, 20], atol=1e-9)


def test_rib_pointlight_profile(tmp_path):
    (tmp_path / "down.ies").write_text(DOWNLIGHT)
    s = load_rib_string('Rotate 90 0 0 1\nLightSource "pointlight" 1 "from" [0 2 0] "intensity" [3] '
                        '"string iesProfile" ["down.ies"]\n'
                        'LightSource "pointlight" 2 "from" [0 2 0] "string iesProfile" ["nope.ies"]',
                        base_dir=str(tmp_path))
    assert list(s.ies) == [0]
    v, h, c, m = s.ies[0]
    assert len(v) == 5 and c.shape == (1, 5)
    # The inverse of a 90-degree turn about z.
    np.testing.assert_allclose(m, [[0, 1, 0], [-1, 0, 0], [0, 0, 1]], atol=1e-12)
    assert any("nope.ies" in w for w in s.warnings)


def _create(s):
    h = C.c_void_p()
    d = s.desc()
    p = abi.make_params(bvh_build="host")
    rc = backend.lib().rt_session_create(C.byref(d), C.byref(p), C.byref(h))
    return rc, backend.lib().rt_last_error().decode()


def test_profile_on_a_non_point_light_refused():
    s = scene.Scene(4, 4)
    s.add_instance(s.add_mesh([[0, 0, 1], [1, 0, 1], [0, 1, 1]], [[0, 1, 2]]),
                   s.add_material(scene.matte((0.5, 0.5, 0.5))))
    li = s.add_distant_light((0, -1, 0), 1.0)
    s.ies[li] = parse_ies(DOWNLIGHT) + (np.eye(3),)
    rc, msg = _create(s)
    assert rc == -1 and "not on a point light" in msg
