"""Sample-range rendering over two gloo ranks on the host: each rank renders
its range with the f64 oracle (standing in for its GPU), the accumulators
are merged by the package's all-reduce, and the result equals one process
rendering the whole range; checkpoint merging likewise."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from rtcuda import abi, scenes
from rtcuda.distributed import (merge_checkpoints, read_checkpoint, render_distributed, sample_range,
                                write_checkpoint)

SPP = 6


def _oracle_accum(scene, params, start, count):
    acc = np.zeros((scene.height * scene.width, 4))
    if count:
        rgb = oracle.OracleScene(scene).render(params, start, start + count)[0]
        acc[:, :3] = rgb
        acc[:, 3] = count
    return acc.reshape(scene.height, scene.width, 4)


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = scenes.cornell_box(8, 8)
        acc = render_distributed(s, abi.make_params(max_depth=4), SPP, sample0=3, render_fn=_oracle_accum)
        np.save(os.path.join(out, f"rank{rank}.npy"), acc)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_sample_ranges_cover_the_frame():
    for spp, world in ((16, 2), (7, 3), (2, 4)):
        ranges = [sample_range(spp, r, world, 5) for r in range(world)]
        assert sum(c for _, c in ranges) == spp
        assert all(ranges[i][0] + ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
        assert ranges[0][0] == 5
    with pytest.raises(ValueError):
        sample_range(4, 2, 2)


def test_two_gloo_ranks_merge_to_the_single_render():
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        a0, a1 = np.load(os.path.join(out, "rank0.npy")), np.load(os.path.join(out, "rank1.npy"))
    s = scenes.cornell_box(8, 8)
    full = _oracle_accum(s, abi.make_params(max_depth=4), 3, SPP)
    assert np.array_equal(a0, a1)
    np.testing.assert_allclose(a0, full, rtol=1e-12, atol=1e-12)
    assert (a0[..., 3] == SPP).all()


def test_checkpoint_merge(tmp_path):
    s = scenes.cornell_box(8, 8)
    p = abi.make_params(max_depth=4)
    parts = []
    for i, (start, count) in enumerate(sample_range(SPP, r, 3) for r in range(3)):
        path = str(tmp_path / f"part{i}.rcu")
        write_checkpoint(path, _oracle_accum(s, p, start, count), count)
        parts.append(path)
    acc, total = merge_checkpoints(parts, str(tmp_path / "merged.rcu"))
    w, h, done, back = read_checkpoint(str(tmp_path / "merged.rcu"))
    assert (w, h, done, total) == (8, 8, SPP, SPP)
    np.testing.assert_allclose(back, _oracle_accum(s, p, 0, SPP), rtol=1e-12, atol=1e-12)
    write_checkpoint(str(tmp_path / "odd.rcu"), np.zeros((4, 8, 4)), 1)
    with pytest.raises(ValueError):
        merge_checkpoints(parts + [str(tmp_path / "odd.rcu")], str(tmp_path / "bad.rcu"))
