"""Sample-range rendering on the GPU merged through checkpoint files: two
sessions render consecutive sample ranges of a frame, their checkpoints are
merged, and the merged accumulator (loaded back into a session) equals one
session rendering the whole range."""
import numpy as np
import pytest

from rtcuda import PtSession, abi, scenes
from rtcuda.distributed import image_from_accum, merge_checkpoints, sample_range

pytestmark = pytest.mark.gpu


def test_checkpoint_merge_equals_single_render(tmp_path):
    s = scenes.cornell_box(64, 64)
    p = abi.make_params(max_depth=8)
    spp, world = 24, 3
    paths = []
    for r in range(world):
        start, count = sample_range(spp, r, world, sample0=11)
        with PtSession(s, p) as g:
            g.render_samples(start, count)
            path = str(tmp_path / f"range{r}.rcu")
            g.checkpoint_save(path)
            paths.append(path)
    acc, total = merge_checkpoints(paths, str(tmp_path / "merged.rcu"))
    assert total == spp
    with PtSession(s, p) as g:
        g.render_samples(11, spp)
        single = g.sum_and_weight()
    np.testing.assert_allclose(acc, single, rtol=1e-12, atol=1e-12)
    with PtSession(s, p) as g:
        g.checkpoint_load(str(tmp_path / "merged.rcu"))
        np.testing.assert_allclose(g.image(), image_from_accum(single), rtol=1e-6, atol=1e-7)


def test_accum_exr_ranges_merge_like_the_reference(tmp_path):
    # --sample-range A:B on each node writes an accumulation EXR; `render
    # merge` averages them (src/main.rs:363-403, src/output/accum.rs:88-119).
    from rtcuda import accum
    s = scenes.cornell_box(48, 40)
    p = abi.make_params(max_depth=8)
    files = []
    for k, (a, b) in enumerate(((0, 5), (5, 16), (16, 24))):
        with PtSession(s, p) as g:
            g.render_samples(a, b - a)
            f = tmp_path / f"node{k}.exr"
            g.write_accum_exr(f)
            files.append(f)
    merged = accum.merge(files)
    with PtSession(s, p) as g:
        g.render_samples(0, 24)
        whole = g.sum_and_weight()
    want = whole[..., :3] / whole[..., 3:]
    np.testing.assert_allclose(merged, want, rtol=2e-6, atol=1e-6)
    sums = sum(accum.read_accum(f) for f in files)
    np.testing.assert_array_equal(sums[..., 3], whole[..., 3])


def test_metal_checkpoint_format_resumes(tmp_path):
    # RCKP (src/raytracer/metal/renderer.rs:219-254): f32 accumulator; a
    # render resumed from it matches an uninterrupted one to f32 rounding.
    s = scenes.cornell_box(40, 32)
    p = abi.make_params(max_depth=8)
    ck = str(tmp_path / "ck.rckp")
    with PtSession(s, p) as g:
        g.render_samples(0, 8)
        g.checkpoint_save_rckp(ck)
    with PtSession(s, p) as g:
        assert g.checkpoint_load(ck) == 8
        g.render_samples(8, 8)
        resumed = g.sum_and_weight()
    with PtSession(s, p) as g:
        g.render_samples(0, 16)
        whole = g.sum_and_weight()
    np.testing.assert_allclose(resumed, whole, rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(resumed[..., 3], whole[..., 3])
