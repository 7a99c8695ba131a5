"""rtcuda — B200 (sm_100a) wavefront path tracer for render.rs scenes.

Host-side mirror of the reference's GPU backend interface over the C ABI of
librtcuda.so (include/rt_cuda.h): scene in, beauty and AOV framebuffer out,
with per-(pixel, sample) PCG32 seeding. Scenes come from the builder API
(``scene.Scene``) or RIB files (``rib.load_rib``); file textures, IES
profiles and environment maps are read by ``textures``, ``ies`` and
``envmap``.
"""
from . import abi, scene, scenes  # noqa: F401
from .backend import (PtSession, RtError, decode_film, intersect_probe, render_pt,  # noqa: F401
                      render_pt_checkpointed, render_pt_film)
