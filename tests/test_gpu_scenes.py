"""Statistical parity with the f64 oracle on the remaining workloads, at
reduced resolution: the instanced-materials scene (1,000 instances of 4
meshes, GGX / Oren-Nayar / rough-glass materials, 64 point lights through
the light BVH) and a reduced forest (bark + leaf instances with a presence
cutout, hundreds of point lights, fBm terrain)."""
import numpy as np
import pytest

import oracle
from rtcuda import PtSession, abi, scenes

pytestmark = pytest.mark.gpu


def _parity(s, p, spp, mean_tol):
    cpu = oracle.OracleScene(s).render(p, 0, spp)[0].reshape(s.height, s.width, 3) / spp
    with PtSession(s, p) as g:
        g.render_samples(0, spp)
        gpu = g.image()
        st = g.stats()
    mc, mg = cpu.reshape(-1, 3).mean(0), gpu.reshape(-1, 3).mean(0)
    rel = np.abs(mc - mg) / np.maximum(mc, 0.02)
    assert (rel < mean_tol).all(), (mc, mg)
    return st


def test_instanced_materials_parity():
    s = scenes.instanced_materials(48, 27, subdivisions=3, grid=32)
    st = _parity(s, abi.make_params(max_depth=12), 256, 0.05)
    assert st["shadow_rays"] > 0


def test_forest_with_cutouts_parity():
    s = scenes.forest(48, 27, n_trees=3, n_placements=3000, n_lights=200, terrain=64, tree_levels=4, extent=120.0)
    assert any(m["presence"] < 1.0 for m in s.materials)
    _parity(s, abi.make_params(max_depth=10), 64, 0.06)


def test_forest_full_scale_builds_and_renders():
    """772,000 instances, ~1.46M unique triangles: the session builds and a
    low-resolution frame renders without device errors."""
    s = scenes.forest(64, 36)
    assert s.n_instances == 772_001
    with PtSession(s, abi.make_params(max_depth=10)) as g:
        st = g.stats()
        assert st["tlas_nodes"] > 0 and st["triangles"] > 1_000_000
        g.render_samples(0, 4)
        img = g.image()
    assert np.isfinite(img).all() and img.mean() > 0
