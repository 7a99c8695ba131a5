"""The allocation-free ray batch (rt_intersect_batch_noalloc).

Callers that may not allocate device memory once they are set up (a frame
loop with a fixed memory budget, or a host application that owns all device
allocation) use this entry point; its staging lives in a fixed static device
array instead of cudaMalloc'd buffers. It must give the same answers as
rt_intersect_batch, call after call (the shared array keeps the previous
call's contents, so the work counter has to be cleared every time), and must
refuse batches larger than its fixed staging area.

This file is collected last so that a run stopping at the first failure has
already run every other test; it passes alone or after the others.
"""
import ctypes as C

import numpy as np
import pytest

from rtcuda import PtSession, backend, scene, scenes

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536  # RT_NOALLOC_MAX_RAYS in include/rt_cuda.h


def _noalloc(sess, planes, any_hit):
    lib = backend.lib()
    f = lib.rt_intersect_batch_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    n = planes.shape[1]
    prim = np.full(n, 7, dtype=np.uint32)
    inst = np.full(n, 7, dtype=np.uint32)
    t = np.full(n, -1.0, dtype=np.float32)
    rc = f(sess.h, planes.ctypes.data, n, 1 if any_hit else 0, prim.ctypes.data, inst.ctypes.data, t.ctypes.data)
    return rc, prim, inst, t


@pytest.fixture(scope="module")
def cloud_session():
    s = scene.Scene(8, 8)
    s.add_instance(s.add_mesh(*scenes.triangle_cloud_mesh(50_000, seed=21)), s.add_material(scene.matte((0.5,) * 3)))
    with PtSession(s) as g:
        yield g


@pytest.mark.parametrize("any_hit", [False, True])
def test_noalloc_matches_allocating_batch_twice(cloud_session, any_hit):
    g = cloud_session
    for call, seed in enumerate((31, 32)):   # two calls in a row, different rays
        rays = scenes.triangle_cloud_rays(MAX_RAYS if call == 0 else 40_000, seed=seed)
        if any_hit:
            rays[1, :, 3] = 2.0
        rc, prim, inst, t = _noalloc(g, rays, any_hit)
        assert rc == 0, backend.lib().rt_last_error()
        ref_p, ref_i, ref_t = g.intersect(rays, any_hit=any_hit)
        if any_hit:
            assert np.array_equal(prim.astype(bool), ref_p)
        else:
            assert np.array_equal(prim, ref_p) and np.array_equal(inst, ref_i)
            hit = ref_p != 0xFFFFFFFF
            assert np.allclose(t[hit], ref_t[hit], rtol=1e-6, atol=0)
            assert np.isinf(t[~hit]).all()


def test_noalloc_rejects_oversized_batch(cloud_session):
    rays = np.zeros((2, MAX_RAYS + 1, 4), dtype=np.float32)
    rc, _, _, _ = _noalloc(cloud_session, rays, False)
    assert rc == -1
    assert "exceed" in backend.lib().rt_last_error().decode()


def test_noalloc_allocates_nothing(cloud_session):
    """After one warm-up call, further calls leave the device's free memory
    and the session's own device bytes unchanged."""
    import torch
    g = cloud_session
    rays = scenes.triangle_cloud_rays(MAX_RAYS, seed=33)
    rc, _, _, _ = _noalloc(g, rays, False)
    assert rc == 0, backend.lib().rt_last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    held0 = g.stats()["device_bytes"]
    for any_hit in (False, True, False, True, False):
        rc, _, _, _ = _noalloc(g, rays, any_hit)
        assert rc == 0, backend.lib().rt_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert g.stats()["device_bytes"] == held0
