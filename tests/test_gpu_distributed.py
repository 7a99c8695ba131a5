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
