"""Rendering a frame across processes by sample range, and merging the f64
accumulators — the reference's `--sample-range` runs plus `merge`
(src/main.rs:363-403, src/raytracer/output/accum.rs:88-119).

Per-(pixel, sample) seeding makes any split of the sample range exact: rank r
renders its own consecutive samples, and the merged accumulator (radiance
sums and sample weights) is the elementwise sum. No data-path collective
runs while rendering; the one exchange is a sum of the accumulators (an
all-reduce over the process group, or a merge of checkpoint files written by
independent runs).
"""
import struct

import numpy as np

CHECKPOINT_MAGIC = 0x31554352  # "RCU1": rt_checkpoint_save's header word


def sample_range(spp, rank, world, sample0=0):
    """(first sample, count) of `rank` when `spp` samples are split over
    `world` ranks in consecutive blocks (the first spp % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(int(spp), world)
    start = rank * base + min(rank, extra)
    return sample0 + start, base + (1 if rank < extra else 0)


def image_from_accum(acc):
    """(H, W, 3) float32 image: radiance sums divided by the sample weight."""
    acc = np.asarray(acc, dtype=np.float64)
    w = np.maximum(acc[..., 3:4], 1e-300)
    return (acc[..., :3] / w).astype(np.float32)


def merge_accumulators(acc, group=None):
    """Sum an (H, W, 4) f64 accumulator over the ranks of a torch.distributed
    process group (gloo on host memory, NCCL on the current CUDA device)."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(acc, dtype=np.float64))
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def render_distributed(scene, params, spp, sample0=0, render_fn=None, group=None):
    """Render `spp` samples per pixel split over the ranks of `group`; every
    rank returns the merged (H, W, 4) f64 accumulator. `render_fn(scene,
    params, start, count)` renders one rank's range and returns its
    accumulator; by default a GPU session of this package."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    start, count = sample_range(spp, rank, world, sample0)
    if render_fn is None:
        render_fn = _render_gpu
    acc = render_fn(scene, params, start, count)
    return merge_accumulators(acc, group)


def _render_gpu(scene, params, start, count):
    from .backend import PtSession
    with PtSession(scene, params) as s:
        if count:
            s.render_samples(start, count)
        return s.sum_and_weight()


def read_checkpoint(path):
    """(width, height, samples_done, (H, W, 4) f64 accumulator) of a checkpoint
    written by rt_checkpoint_save."""
    with open(path, "rb") as f:
        hdr = f.read(16)
        if len(hdr) != 16:
            raise ValueError(f"{path}: truncated header")
        magic, w, h, done = struct.unpack("<4I", hdr)
        if magic != CHECKPOINT_MAGIC:
            raise ValueError(f"{path}: not a checkpoint (magic {magic:#x})")
        data = np.frombuffer(f.read(), dtype="<f8")
    if data.size != w * h * 4:
        raise ValueError(f"{path}: {data.size} values for a {w}x{h} accumulator")
    return w, h, done, data.reshape(h, w, 4).copy()


def write_checkpoint(path, acc, samples_done):
    """Write an accumulator in rt_checkpoint_save's format (loadable by
    rt_checkpoint_load)."""
    acc = np.ascontiguousarray(acc, dtype="<f8")
    h, w = acc.shape[:2]
    with open(path, "wb") as f:
        f.write(struct.pack("<4I", CHECKPOINT_MAGIC, w, h, int(samples_done)))
        f.write(acc.tobytes())


def merge_checkpoints(paths, out_path):
    """Sum the accumulators of checkpoints from independent sample-range runs
    of one frame (the reference's `merge`); the merged file records the total
    samples. Frames of different sizes are rejected."""
    total, acc, size = 0, None, None
    for p in paths:
        w, h, done, a = read_checkpoint(p)
        if size is None:
            size, acc = (w, h), a
        elif (w, h) != size:
            raise ValueError(f"{p}: {w}x{h} frame, expected {size[0]}x{size[1]}")
        else:
            acc = acc + a
        total += done
    if acc is None:
        raise ValueError("no checkpoints to merge")
    write_checkpoint(out_path, acc, total)
    return acc, total
