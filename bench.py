"""Benchmark: the large-scale forest workload on B200.

Workload (one step): one full frame of the procedural forest -- 20 seeded
trees (bark + leaf meshes, ~46k triangles each, leaves with a presence
cutout of 0.5) placed as 772,000 instances on a 1 km^2 fBm terrain, 1,200
point lights through the light BVH -- rendered at 3840x2160 with 32 samples
per pixel, max depth 10, Russian roulette from depth 3: 265,420,800 camera
samples per step, plain (unguided) path tracing.

Printed (one JSON line on rank 0):
  value      Msamples/s of the whole job, scene and path state resident in HBM
             (device time, CUDA events on the session stream, max over ranks);
  e2e        the same metric through the C ABI's render call a user makes
             (rt_session_create from host arrays, incl. the device BVH build,
             + rt_render_samples of the 32 passes + rt_read_image to host),
             host<->device copies included;
  roofline   the closest-hit (extend) kernel: algorithmic bytes per
             extension ray (reference binary BVH: 32 B per node visit, 48 B
             per triangle test, 48 B per instance visit, 48 B ray in/out,
             counted by the f64 oracle on a pixel sample of the same frame)
             x extension rays per launch / launch time, against the measured
             HBM copy bandwidth;
  cpu_baseline  the f64 oracle (C++ restatement of the reference's CPU path
             tracer, all host threads) on a bounded pixel sample of the frame.
  workloads  the other configurations: the 1M-triangle cloud at 1920x1080 x
             16 spp and its 4,194,304-ray closest-hit / any-hit batches, the
             Cornell box 256^2 x 16 spp, instanced materials 1920x1080 x 64
             spp (device Msamples/s and Mrays/s).
  guided_equal_time  the learned-proposal workload: two 4x3x3 rooms joined by
             a 0.2x2.0 opening, the light in the unseen room, 1280x720, max
             depth 16. A fresh guided session renders GUIDED_SPP passes from
             an untrained network (online training included in its time); a
             plain session renders as many passes as fit in the same device
             time. Both are scored by relMSE against a high-spp GPU render
             (all pixels) and against the f64 CPU oracle on a strided pixel
             subset, with a confidence interval over the pixels.
  guided_forest  the forest's guided-vs-plain comparison at reduced size.

`--impl reference` times the reference arm instead: the reference's CPU path
(its Rust build is unavailable here, so the f64 C++ restatement of
src/raytracer/pt/*) on the host cores, on a bounded pixel sample of the same
frame each step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "render.rs_b200"))

METRIC = "Msamples/s at 1 B200; equal-time relMSE guided vs plain PT vs f64 CPU oracle"
UNIT = "Msamples/s"
# The headline workload: the forest at its configured size.
WIDTH, HEIGHT, SPP, MAX_DEPTH = 3840, 2160, 32, 10
WORKLOAD = "forest_772k_instances_1200_lights_3840x2160_32spp_depth10"
CONFIG = {"workload": WORKLOAD, "width": WIDTH, "height": HEIGHT, "spp": SPP, "max_depth": MAX_DEPTH,
          "rr_start": 3, "instances": 772_001, "trees": 20, "point_lights": 1200, "presence_cutouts": True,
          "guided": False, "l2_flush": "256 MB write before every step; scene + path state > L2"}
def config_for(world):
    """The `config` both arms print (the driver compares them)."""
    return dict(CONFIG, parallelism=f"replica-sample-ranges x{world}", accumulator="f64")


# The traversal-stress workload (a `workloads` entry).
CLOUD_W, CLOUD_H, CLOUD_SPP, CLOUD_DEPTH = 1920, 1080, 16, 8
N_TRIS, N_RAYS = 1_000_000, 4_194_304


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_sample(o_s, scene, params, n_pixels, offset=0, threads=0):
    """The f64 oracle (all host threads unless `threads`) on `n_pixels`
    strided pixels of the frame at SPP samples each: (Msamples/s, sample
    description, cores, per-sample traversal work, seconds)."""
    npix = scene.width * scene.height
    stride = max(1, npix // n_pixels)
    pixels = np.arange(offset % stride, npix, stride, dtype=np.uint32)[:n_pixels]
    t0 = time.perf_counter()
    _, _, counts = o_s.render(params, 0, SPP, pixels=pixels, threads=threads)
    el = time.perf_counter() - t0
    samples = len(pixels) * SPP
    cores = threads if threads > 0 else os.cpu_count()
    ext, sh = int(counts[0]), int(counts[1])
    # Reference binary-BVH bytes (32 B / node visit, 48 B / triangle test,
    # 48 B / instance visit, 48 B ray in + hit out) of the extension rays,
    # per camera sample; presence skips re-trace as extension rays there.
    ext_bytes = 32.0 * counts[2] + 48.0 * counts[3] + 48.0 * counts[4] + 48.0 * ext
    work = {"ext_rays_per_sample": ext / samples, "shadow_segments_per_sample": sh / samples,
            "ext_bytes_per_sample": ext_bytes / samples, "ext_bytes_per_ray": ext_bytes / max(ext, 1),
            "node_visits_per_ext_ray": counts[2] / max(ext, 1), "tri_tests_per_ext_ray": counts[3] / max(ext, 1),
            "instance_visits_per_ext_ray": counts[4] / max(ext, 1)}
    return (samples / el / 1e6, f"{len(pixels)} pixels (every {stride}th) x {SPP} spp of the frame", cores, work,
            el)


GUIDED_W, GUIDED_H, GUIDED_SPP, GUIDED_DEPTH = 1280, 720, 2048, 16

# DRAM bytes (read + write) per extension ray of k_extend on the forest, from
# one ncu capture of all 10 k_extend launches of a 1280x720 pass of the same
# scene (849.6 MB for 1,985,150 extension rays; 1 metric pass):
#   ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum,lts__t_bytes.sum
#       --clock-control none -k regex:"k_extend" -s 10 -c 10
#       python bench.py --mode scene --scene forest --res 1280x720 --steps 1 --warmup 1
# A 3840x2160 launch is scaled from it by its rays; per-ray traffic falls as
# the frame grows (582 B per ray over the first waves at 640x360), so the
# scaled figure is an upper bound.
EXTEND_DRAM_BYTES_PER_RAY = 849.6e6 / 1_985_150
EXTEND_DRAM_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the 10 k_extend launches of a "
                      "1280x720 forest pass (428 B per extension ray), scaled by the rays per launch")


def rel_mse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def ratio_ci(plain, guided, ref, z=1.96):
    """relMSE(plain) / relMSE(guided) against `ref` with a confidence
    interval over the pixels (delta method on the ratio of the per-pixel
    means; pixels are independent)."""
    den = ref.reshape(-1, 3) ** 2 + 1e-2
    a = ((plain.reshape(-1, 3) - ref.reshape(-1, 3)) ** 2 / den).mean(1)
    b = ((guided.reshape(-1, 3) - ref.reshape(-1, 3)) ** 2 / den).mean(1)
    n = len(a)
    ma, mb = a.mean(), b.mean()
    r = ma / mb
    cov = np.cov(a, b)
    var = (cov[0, 0] / mb ** 2 + ma ** 2 * cov[1, 1] / mb ** 4 - 2 * ma * cov[0, 1] / mb ** 3) / n
    h = z * float(np.sqrt(max(var, 0.0)))
    return float(r), [float(r - h), float(r + h)]


def equal_time_plain(scene, params, budget_ms, first=64):
    """Plain render for the same device time as `budget_ms`: `first` passes,
    then whole slabs at a time (the session's own slab size, so no pass runs
    in an undersized slab) until the summed device time reaches the budget.
    Returns (image, passes, device ms)."""
    from rtcuda import PtSession
    with PtSession(scene, params) as g:
        g.render_samples(0, first)
        st = g.stats()
        done, ms = first, st["total_ms"]
        slab = max(1, -(-first // max(1, st["slabs"])))
        while ms < budget_ms:
            g.render_samples(done, slab)
            done += slab
            ms += g.stats()["total_ms"]
        return g.image(), done, ms


def guided_equal_time(ref_spp=16384, cpu_pixels=4096, cpu_spp=65536):
    """Equal-time relMSE of guided vs plain path tracing on the two-room scene.
    The GPU reference is the mean of two independent halves A and B; its own
    error, mean((A - B)^2 / (ref^2 + 1e-2)) / 4, is reported and subtracted
    in the `*_corrected` figures (it adds to both estimators' relMSE)."""
    from rtcuda import PtSession, abi, scenes
    s = scenes.two_rooms(GUIDED_W, GUIDED_H)
    plain_p = abi.make_params(max_depth=GUIDED_DEPTH)
    guided_p = abi.make_params(max_depth=GUIDED_DEPTH, guided=True, guide_fraction=0.5)
    halves = []
    for h in range(2):                                     # high-spp GPU reference, two halves
        with PtSession(s, plain_p) as g:
            g.render_samples((1 << 24) + h * ref_spp, ref_spp // 2)
            halves.append(g.image())
    ref = 0.5 * (halves[0] + halves[1])
    ref_err = float(np.mean((halves[0] - halves[1]) ** 2 / (ref ** 2 + 1e-2))) / 4.0
    with PtSession(s, guided_p) as g:                      # warm-up of the code paths only
        g.render_samples(1 << 23, 2)
    with PtSession(s, guided_p) as g:
        g.render_samples(0, GUIDED_SPP)
        st = g.stats()
        guided_ms = st["total_ms"]
        guided = g.image()
    plain, plain_spp, plain_ms = equal_time_plain(s, plain_p, guided_ms)
    per_spp = plain_ms / plain_spp
    out = {"scene": f"two_rooms_{GUIDED_W}x{GUIDED_H}_depth{GUIDED_DEPTH}", "guided_spp": GUIDED_SPP,
           "guided_ms": round(guided_ms, 2), "guide_steps": st["guide_steps"], "plain_spp": plain_spp,
           "plain_ms": round(plain_ms, 2), "plain_ms_per_spp": round(per_spp, 4),
           "gpu_reference_spp": ref_spp}
    e_p, e_g = rel_mse(plain, ref), rel_mse(guided, ref)
    out["ratio_vs_gpu_ref_ci95"] = ratio_ci(plain, guided, ref)[1]
    out.update({"relmse_plain_vs_gpu_ref": e_p, "relmse_guided_vs_gpu_ref": e_g, "ratio_vs_gpu_ref": e_p / e_g,
                "gpu_ref_relmse": ref_err, "relmse_plain_corrected": e_p - ref_err,
                "relmse_guided_corrected": e_g - ref_err, "ratio_corrected": (e_p - ref_err) / (e_g - ref_err),
                "guide_steps_per_pass": st["guide_steps"] / GUIDED_SPP})
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle  # test infrastructure: the f64 reference pixels
        npix = GUIDED_W * GUIDED_H
        pix = np.arange(npix // (2 * cpu_pixels), npix, npix // cpu_pixels, dtype=np.uint32)[:cpu_pixels]
        t0 = time.perf_counter()
        acc = oracle.OracleScene(s).render(plain_p, 1 << 25, (1 << 25) + cpu_spp, pixels=pix)[0]
        cref = acc / cpu_spp  # (n, 3) radiance sums of the sampled pixels
        el = time.perf_counter() - t0
        gp, gg = plain.reshape(-1, 3)[pix], guided.reshape(-1, 3)[pix]
        c_p, c_g = rel_mse(gp, cref), rel_mse(gg, cref)
        r, ci = ratio_ci(gp, gg, cref)
        out.update({"relmse_plain_vs_f64": c_p, "relmse_guided_vs_f64": c_g, "ratio_vs_f64": r,
                    "ratio_vs_f64_ci95": ci,
                    "f64_reference": f"oracle, {len(pix)} strided pixels x {cpu_spp} spp ({el:.1f} s)"})
    except Exception as exc:  # the oracle is optional on a box without it
        out["f64_reference"] = f"unavailable: {exc}"
    return out


def load_tensor_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)["bf16_tflops"], "measured"
    except Exception:
        return 1590.0, "fallback"


GUIDE_FWD_FLOP = 2 * (48 * 64 + 64 * 64 + 64 * 64 + 64 * 48)   # MLP 48-64-64-64-48 per record


def guide_network_rate(n_infer=1 << 20, n_train=1 << 16, reps=20):
    """The learned proposal's tcgen05 MLP alone, device-resident records:
    inference of 2^20 records (hash-grid encode + forward) and training
    steps of 2^16 records (encode, forward, backward, gradient reduction,
    hash-grid backward, Adam), CUDA events on one stream. FLOP/s count the
    MLP's algorithmic FLOPs (forward 28,672 per record; a training step
    forward + backward = 3x) against the measured dense bf16 peak."""
    import ctypes
    import torch
    from rtcuda import guide as G
    peak, kind = load_tensor_peak()
    g = G.Guide((-1, -1, -1), (1, 1, 1), seed=3, lr=1e-2)
    L = G._g()
    rng = np.random.default_rng(1)
    rec = np.zeros((n_infer, 16), np.float32)
    rec[:, 0:3] = rng.uniform(-1, 1, (n_infer, 3))
    for a, b in ((3, 6), (6, 9), (9, 12)):
        v = rng.normal(size=(n_infer, 3))
        rec[:, a:b] = v / np.linalg.norm(v, axis=1, keepdims=True)
    rec[:, 12] = rng.uniform(0.0, 2.0, n_infer)
    d_rec = torch.from_numpy(rec).cuda()
    d_out = torch.empty((n_infer, 48), dtype=torch.float32, device="cuda")
    st = torch.cuda.Stream()
    sp = ctypes.c_void_p(st.cuda_stream)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(reps):
            fn()
        b.record(st)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    infer_ms = timed(lambda: G._check(L.rt_guide_infer_device(g.h, d_rec.data_ptr(), n_infer, d_out.data_ptr(), sp)))
    train_ms = timed(lambda: G._check(L.rt_guide_train_step_device(g.h, d_rec.data_ptr(), n_train, None, sp)))
    g.close()
    inf_tf = n_infer * GUIDE_FWD_FLOP / (infer_ms * 1e-3) / 1e12
    tr_tf = 3 * n_train * GUIDE_FWD_FLOP / (train_ms * 1e-3) / 1e12
    return {"inference_records": n_infer, "inference_ms": round(infer_ms, 4), "inference_tflops": inf_tf,
            "inference_frac": inf_tf / peak, "train_records": n_train, "train_step_ms": round(train_ms, 4),
            "train_tflops": tr_tf, "train_frac": tr_tf / peak, "peak_tflops": peak, "peak_kind": kind,
            "flop_per_record_forward": GUIDE_FWD_FLOP}


def other_workloads(flush, stream):
    """Device throughput of the other configurations at their configured
    size: the 1M-triangle cloud at 1920x1080 x 16 spp (depth 8) and its
    4,194,304-ray closest-hit / any-hit batches (L2 flushed before each
    batch), the Cornell box 256^2 x 16 spp (depth 8), instanced materials
    1920x1080 x 64 spp (depth 12), the media Cornell box 512^2 x 16 spp (fog,
    an fBm cloud, absorbing glass, a subsurface sphere; 64 bounces, the
    reference's depth with media), the furball 960x480 x 16 spp (20,000
    b-spline strands of Marschner hair, 480,000 segments), the Cornell box
    with motion blur (a moving box, a deforming sheet and camera motion) and
    with all of it static, 512^2 x 16 spp, and the pattern-cutout screens
    512x384 x 16 spp. One warm-up pass, then one timed render call (device
    time from the session's events); scene build excluded."""
    import torch
    from rtcuda import PtSession, abi, scenes
    out = {}
    cases = [("triangle_cloud_1M_1920x1080_16spp_depth8", lambda: scenes.triangle_cloud(CLOUD_W, CLOUD_H, N_TRIS),
              scenes.TRIANGLE_CLOUD, CLOUD_SPP),
             ("cornell_256x256_16spp_depth8", lambda: scenes.cornell_box(), scenes.CORNELL, 16),
             ("instanced_materials_1920x1080_64spp_depth12", lambda: scenes.instanced_materials(),
              scenes.INSTANCED_MATERIALS, 64),
             ("media_cornell_512x512_16spp_depth64", lambda: scenes.media_cornell(512, 512),
              dict(max_depth=8, rr_start=3), 16),
             ("furball_20k_strands_960x480_16spp_depth8", lambda: scenes.furball(960, 480, 20_000),
              dict(max_depth=8, rr_start=3), 16),
             ("motion_cornell_512x512_16spp_depth8", lambda: scenes.motion_cornell(512, 512), scenes.CORNELL, 16),
             ("motion_cornell_static_512x512_16spp_depth8",
              lambda: scenes.motion_cornell(512, 512, transform=False, deform=False, camera=False), scenes.CORNELL,
              16),
             ("pattern_cutouts_512x384_16spp_depth8", lambda: scenes.pattern_cutouts(512, 384), scenes.CORNELL, 16)]
    for name, make, cfg, spp in cases:
        t0 = time.perf_counter()
        s = make()
        p = abi.make_params(max_depth=cfg["max_depth"], rr_start=cfg["rr_start"])
        with PtSession(s, p) as g:
            build_s = time.perf_counter() - t0
            g.render_samples(1 << 20, 1)
            g.render_samples(0, spp)
            st = g.stats()
            ms = st["total_ms"]
            out[name] = {"Msamples_per_s": st["samples"] / ms / 1e3, "ms": round(ms, 2), "spp": spp,
                         "Mrays_per_s": (st["extension_rays"] + st["shadow_rays"]) / ms / 1e3,
                         "extend_ms": round(st["extend_ms"], 2), "extension_rays": st["extension_rays"],
                         "triangles_effective": s.triangle_count(), "instances": s.n_instances,
                         "build_and_upload_s": round(build_s, 2)}
            if name.startswith("triangle_cloud"):
                out[name]["traversal"] = traversal_batches(g, flush)
    return out


def traversal_batches(sess, flush, reps=5):
    """The 4,194,304-ray closest-hit and any-hit batches into the session's
    scene from HBM (CUDA events on the session stream, L2 flushed before
    each batch)."""
    import torch
    from rtcuda import scenes
    stream = torch.cuda.ExternalStream(sess.stream())
    d_rays = torch.from_numpy(scenes.triangle_cloud_rays(N_RAYS)).cuda()
    prim = torch.empty(N_RAYS, dtype=torch.int32, device="cuda")
    inst = torch.empty_like(prim)
    tt = torch.empty(N_RAYS, dtype=torch.float32, device="cuda")
    trav = {}
    for any_hit, name in ((0, "closest_hit"), (1, "any_hit")):
        for _ in range(3):
            sess.intersect_device(d_rays.data_ptr(), N_RAYS, any_hit, prim.data_ptr(), inst.data_ptr(),
                                  tt.data_ptr(), sess.stream())
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        tot = 0.0
        for _ in range(reps):
            with torch.cuda.stream(stream):
                flush.zero_()
            a.record(stream)
            sess.intersect_device(d_rays.data_ptr(), N_RAYS, any_hit, prim.data_ptr(), inst.data_ptr(),
                                  tt.data_ptr(), sess.stream())
            b.record(stream)
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        tms = tot / reps
        trav[name] = {"ms": round(tms, 3), "Mrays_per_s": N_RAYS / tms / 1e3}
    return trav


def guided_forest(width=480, height=270, budget=128, ref_spp=512):
    """The large-scale workload's guided-vs-plain comparison, reduced: the
    forest (772,001 instances, 1,200 point lights, depth 10) at
    `width` x `height`, `budget` guided passes from an untrained network
    against plain passes in the same device time, relMSE against a GPU
    reference of `ref_spp` passes (two halves; its own noise is removed in
    `ratio_corrected`). The comparison against a 4,096-spp f64 crop is hours
    of CPU time and is not run; `--mode guided-forest --res 3840x2160` runs
    this one at the full frame size."""
    from rtcuda import PtSession, abi, scenes
    s = scenes.forest(width, height)
    cfg = scenes.FOREST
    plain_p = abi.make_params(max_depth=cfg["max_depth"], rr_start=cfg["rr_start"])
    guided_p = abi.make_params(max_depth=cfg["max_depth"], rr_start=cfg["rr_start"], guided=True)
    halves = []
    for h in range(2):
        with PtSession(s, plain_p) as g:
            g.render_samples((1 << 24) + h * ref_spp, ref_spp // 2)
            halves.append(g.image())
    ref = 0.5 * (halves[0] + halves[1])
    ref_err = float(np.mean((halves[0] - halves[1]) ** 2 / (ref ** 2 + 1e-2))) / 4.0
    with PtSession(s, guided_p) as g:
        g.render_samples(0, budget)
        guided_ms = g.stats()["total_ms"]
        guided = g.image()
    plain, plain_spp, plain_ms = equal_time_plain(s, plain_p, guided_ms, first=min(64, max(1, budget // 8)))
    e_p, e_g = rel_mse(plain, ref), rel_mse(guided, ref)
    return {"scene": f"forest_{width}x{height}_depth{cfg['max_depth']}", "guided_spp": budget,
            "guided_ms": round(guided_ms, 1), "plain_spp": plain_spp, "plain_ms": round(plain_ms, 1),
            "gpu_reference_spp": ref_spp, "relmse_plain": e_p, "relmse_guided": e_g, "ratio": e_p / e_g,
            "ratio_ci95": ratio_ci(plain, guided, ref)[1],
            # Plain's last slab overshoots the guided time a little; relMSE
            # falls as 1/time, so this scales plain's error to the guided time.
            "ratio_time_scaled": e_p * plain_ms / guided_ms / e_g, "gpu_ref_relmse": ref_err,
            "ratio_corrected": (e_p - ref_err) / (e_g - ref_err) if e_g > ref_err else None}


def run_reference(args):
    """Reference arm: the reference's CPU path (its f64 C++ restatement) on
    the host cores, each step a bounded pixel sample of the same frame."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the reference arm runs the oracle by design
    from rtcuda import abi, scenes
    scene = scenes.forest(WIDTH, HEIGHT)
    params = abi.make_params(max_depth=MAX_DEPTH, rr_start=3)
    o_s = oracle.OracleScene(scene)
    vals, secs, sample, cores = [], [], "", os.cpu_count()
    for i in range(args.warmup + args.steps):
        v, sample, cores, _, el = oracle_sample(o_s, scene, params, REF_PIXELS_PER_STEP, offset=i)
        if i >= args.warmup:
            vals.append(v)
            secs.append(el)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs),
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_for(int(os.environ.get("WORLD_SIZE", str(args.gpus)))),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"per step: {sample}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference is Rust (no toolchain here): its CPU path restated in C++ f64 (oracle/)"}
    print(json.dumps(line), flush=True)
    return 0


REF_PIXELS_PER_STEP = 384   # x 32 spp: a few seconds of the oracle per step on the forest


def run_traversal(args):
    """Closest-hit then any-hit batches over the triangle cloud, `args.rays`
    rays each, device-resident; one JSON line with per-launch times."""
    import torch
    from rtcuda import PtSession, abi, scenes
    from rtcuda.scene import Scene, matte
    s = Scene(8, 8)
    s.add_instance(s.add_mesh(*scenes.triangle_cloud_mesh(N_TRIS)), s.add_material(matte((0.5, 0.5, 0.5))))
    sess = PtSession(s, abi.make_params(max_depth=MAX_DEPTH, max_paths=64))
    stream = torch.cuda.ExternalStream(sess.stream())
    rays = torch.from_numpy(scenes.triangle_cloud_rays(args.rays)).cuda()
    n = args.rays
    prim = torch.empty(n, dtype=torch.int32, device="cuda")
    inst = torch.empty_like(prim)
    tt = torch.empty(n, dtype=torch.float32, device="cuda")
    out = {"mode": "traversal", "rays": n}
    for any_hit, name in ((0, "closest_hit"), (1, "any_hit")):
        for _ in range(args.warmup):
            sess.intersect_device(rays.data_ptr(), n, any_hit, prim.data_ptr(), inst.data_ptr(), tt.data_ptr(),
                                  sess.stream())
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            sess.intersect_device(rays.data_ptr(), n, any_hit, prim.data_ptr(), inst.data_ptr(), tt.data_ptr(),
                                  sess.stream())
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / max(args.steps, 1)
        out[name] = {"ms": ms, "Mrays_per_s": n / ms / 1e3}
    print(json.dumps(out), flush=True)
    sess.close()
    return 0


def run_guided(args):
    """The learned-proposal workload alone (for profiler captures): a fresh
    guided session on the 1280x720 two-room scene renders `args.steps` sample
    passes (slabs grow 1, 2, 4 passes), after `args.warmup` passes in a
    throwaway session; one JSON line with device times from the session."""
    from rtcuda import PtSession, abi, scenes
    s = scenes.two_rooms(GUIDED_W, GUIDED_H)
    p = abi.make_params(max_depth=GUIDED_DEPTH, guided=True, guide_fraction=0.5)
    if args.warmup:
        with PtSession(s, p) as g:
            g.render_samples(1 << 23, args.warmup)
    with PtSession(s, p) as g:
        g.render_samples(0, args.steps)
        st = g.stats()
    print(json.dumps({"mode": "guided", "scene": f"two_rooms_{GUIDED_W}x{GUIDED_H}_depth{GUIDED_DEPTH}",
                      "spp": args.steps, "ms": st["total_ms"], "ms_per_spp": st["total_ms"] / max(args.steps, 1),
                      "guide_steps": st["guide_steps"], "kernel_launches": st["kernel_launches"]}), flush=True)
    return 0


def run_scene(args):
    """One named scene alone (for profiler captures): `--scene`, `--res WxH`,
    `args.warmup` passes in a throwaway call, then `args.steps` passes;
    one JSON line with the session's device-timed stats."""
    from rtcuda import PtSession, abi, scenes
    w, h = (int(v) for v in args.res.split("x"))
    make = {"cornell": (scenes.cornell_box, scenes.CORNELL), "cloud": (scenes.triangle_cloud, scenes.TRIANGLE_CLOUD),
            "instanced": (scenes.instanced_materials, scenes.INSTANCED_MATERIALS),
            "two_rooms": (scenes.two_rooms, scenes.TWO_ROOMS), "forest": (scenes.forest, scenes.FOREST),
            "media": (scenes.media_cornell, dict(max_depth=8, rr_start=3)),
            "furball": (scenes.furball, dict(max_depth=8, rr_start=3))}
    gen, cfg = make[args.scene]
    s = gen(w, h)
    p = abi.make_params(max_depth=cfg["max_depth"], rr_start=cfg["rr_start"])
    with PtSession(s, p) as g:
        if args.warmup:
            g.render_samples(1 << 20, args.warmup)
        g.render_samples(0, args.steps)
        st = g.stats()
    st["Msamples_per_s"] = st["samples"] / st["total_ms"] / 1e3
    print(json.dumps({"mode": "scene", "scene": args.scene, "res": args.res, **st}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--scene", default="forest",
                    help="--mode scene: cornell, cloud, instanced, two_rooms, forest, media, furball")
    ap.add_argument("--res", default="640x360", help="--mode scene: frame size WxH")
    ap.add_argument("--mode", default="full", choices=["full", "traversal", "guided", "scene", "guided-forest"],
                    help="traversal: only the closest/any-hit ray batches; guided: only the learned-proposal "
                         "workload; scene: one named scene (all for profiler captures); guided-forest: the "
                         "forest's equal-time guided-vs-plain comparison at --res with --steps guided passes "
                         "and a --ref-spp GPU reference")
    ap.add_argument("--ref-spp", type=int, default=512, help="--mode guided-forest: passes of the GPU reference")
    ap.add_argument("--rays", type=int, default=N_RAYS)
    ap.add_argument("--no-guided", action="store_true", help="skip the guided equal-time comparisons")
    ap.add_argument("--no-workloads", action="store_true", help="skip the other configurations")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "traversal":
        return run_traversal(args)
    if args.mode == "guided":
        return run_guided(args)
    if args.mode == "scene":
        return run_scene(args)
    if args.mode == "guided-forest":
        w, h = (int(v) for v in args.res.split("x"))
        print(json.dumps({"mode": "guided-forest", **guided_forest(w, h, args.steps, args.ref_spp)}), flush=True)
        return 0

    import torch
    import torch.distributed as dist
    from rtcuda import PtSession, abi, scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)

    scene = scenes.forest(WIDTH, HEIGHT)
    params = abi.make_params(max_depth=MAX_DEPTH, rr_start=3)
    sess = PtSession(scene, params)
    stream = torch.cuda.ExternalStream(sess.stream(), device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    # Weak scaling: every rank renders its own 32-pass frames of the same
    # view (sample ranges offset by rank, as --sample-range partitions the
    # reference's render), so per-GPU work is fixed as ranks are added.
    def step(i):
        with torch.cuda.stream(stream):
            flush.zero_()
        sess.render_samples((rank * 1_000_000 + i * SPP) % (1 << 31), SPP)

    for i in range(args.warmup):
        step(i)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ext_ms = launches = ext_launches = samples = 0.0
    ext_rays = sh_rays = 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
        st = sess.stats()
        ext_ms += st["extend_ms"]
        ext_rays += st["extension_rays"]
        sh_rays += st["shadow_rays"]
        samples += st["samples"]
        ext_launches += st["slabs"] * st["waves"]
        launches += st["kernel_launches"] + 1   # + the L2 flush
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    samples_per_step = WIDTH * HEIGHT * SPP
    value = samples_per_step * args.steps * world / (ms_max / 1e3) / 1e6
    last = sess.stats()
    sess.close()

    # End to end through the C ABI: host scene arrays in (the session
    # uploads them and builds the BVHs on the device), 32 passes, host image
    # out; one session at a time, as a caller rendering frame after frame.
    e2e_ms = []
    h2d = sum(p.nbytes + i.nbytes + (n.nbytes if n is not None else 0) for p, i, n in scene.meshes) + \
        scene.instance_array().nbytes
    d2h = WIDTH * HEIGHT * 3 * 4
    for i in range(args.e2e_steps):
        barrier()
        t0 = time.perf_counter()
        with PtSession(scene, params) as s2:
            s2.render_samples(rank * 1000 + 7 + i * SPP, SPP)
            s2.image()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    et = torch.tensor([max(e2e_ms) if e2e_ms else 0.0], device=dev)
    if world > 1:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e_val = samples_per_step * world / (float(et.item()) / 1e3) / 1e6 if e2e_ms else None

    result = None
    if rank == 0:
        peak, peak_kind = load_peaks()
        cpu = roof = None
        if not args.no_cpu_baseline and world == 1:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle  # test infrastructure: the CPU baseline and the work counter
            o_s = oracle.OracleScene(scene)
            v, sample, cores, work, el = oracle_sample(o_s, scene, params, 2048)
            o_s.close()
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                   "seconds": round(el, 2)}
            launches_ext = max(1.0, ext_launches)
            # Bytes per extension ray (the reference's binary BVH, counted by
            # the oracle) x the extension rays a launch traces.
            alg_bytes = work["ext_bytes_per_ray"] * ext_rays
            achieved = alg_bytes / (ext_ms / 1e3) / 1e9
            # The same work counted per camera sample: a GPU ray passes the
            # cutouts it does not stop at inside one traversal, where the
            # reference traces a new ray after each, so it covers the work of
            # several reference rays.
            per_sample = work["ext_bytes_per_sample"] * samples / (ext_ms / 1e3) / 1e9
            roof = {"kernel": "k_extend (closest hit, 8-wide BVH, cutouts decided in traversal)", "bound": "hbm",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": EXTEND_DRAM_BYTES_PER_RAY * ext_rays / launches_ext,
                    "traffic_source": EXTEND_DRAM_SOURCE,
                    "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg_bytes / launches_ext,
                    "rays_per_launch": ext_rays / launches_ext, "launch_ms": ext_ms / launches_ext,
                    "launches": int(launches_ext), "reference_work": work,
                    "gpu_extension_rays_per_sample": ext_rays / max(samples, 1),
                    "achieved_per_sample_normalised": per_sample}
        workloads = None
        if not args.no_workloads and world == 1:
            workloads = other_workloads(flush, stream)
        guided = forest_guided = network = None
        if not args.no_guided and world == 1:
            network = guide_network_rate()
            guided = guided_equal_time()
            forest_guided = guided_forest()
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_for(world),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": d2h,
                    "ms": max(e2e_ms) if e2e_ms else None, "ms_each": [round(v, 2) for v in e2e_ms]},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            "gpu_launches": int(launches),
            "Mrays_per_s": (ext_rays + sh_rays) / (ms_max / 1e3) / 1e6,
            "rays_per_step": {"extension": ext_rays // max(args.steps, 1), "shadow": sh_rays // max(args.steps, 1)},
            "stage_ms_last_step": {"extend": round(last["extend_ms"], 1), "shade": round(last["shade_ms"], 1),
                                   "shadow": round(last["shadow_ms"], 1), "total": round(last["total_ms"], 1)},
            "workloads": workloads,
            "guided_equal_time": guided,
            "guided_forest": forest_guided,
            "guide_network": network,
        }
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
