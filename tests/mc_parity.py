"""Monte Carlo parity of a GPU render with the f64 oracle.

The tolerance the path tracer is held to: the GPU image's relMSE against a
high-spp oracle render lies within the Monte Carlo confidence interval of
the relMSE that an independent oracle render at the same spp has against
the same reference, and the two same-spp images have the same mean.

With G (GPU) and O (oracle) rendered from disjoint sample ranges at n spp
and R (oracle) from a third range at N >> n spp, per pixel p

    e_G,p = mean_c (G_pc - R_pc)^2 / (R_pc^2 + EPS),   e_O,p likewise.

If G and O follow the same distribution, E[e_G,p - e_O,p] = 0 (R's own
noise adds to both), and the pixels are independent, so the mean of
d_p = e_G,p - e_O,p over the pixels is within z * sd(d) / sqrt(#pixels) of
zero.

Bias is checked on a paired render: P, the oracle over the GPU's own sample
range. The GPU's u32 random streams equal the oracle's (only their
conversion to floats and the arithmetic precision differ), so G_p - P_p is
zero except where a path took another turn; its per-channel mean over the
pixels must lie within z * sd / sqrt(#pixels) of zero, which resolves a
systematic error far smaller than the noise of either image (down to a
floor of 1e-4 of the mean). Renders are
deterministic for their seeds, so a check either always passes or always
fails.
"""
import numpy as np

EPS = 1e-2       # relMSE denominator offset, ref^2 + EPS
Z = 3.0          # two-sided ~99.7% interval
BIAS_FLOOR = 1e-4  # smallest bias bound, relative to the image mean


def compare(gpu, ora, ref, paired=None, z=Z):
    """gpu, ora, ref: (n_pixels, 3) per-pixel means of G, O and R; paired:
    P on the same pixels (None: the bias check uses O). Returns the
    figures; `ok` is True when the relMSE difference and the mean difference
    of every channel lie inside their intervals."""
    gpu, ora, ref = (np.asarray(a, np.float64).reshape(-1, 3) for a in (gpu, ora, ref))
    den = ref ** 2 + EPS
    e_g = ((gpu - ref) ** 2 / den).mean(1)
    e_o = ((ora - ref) ** 2 / den).mean(1)
    n = len(e_g)
    d = e_g - e_o
    half = z * d.std(ddof=1) / np.sqrt(n)
    other = ora if paired is None else np.asarray(paired, np.float64).reshape(-1, 3)
    diff = gpu - other
    bias = diff.mean(0)
    # A floor of 1e-4 of the mean: paired renders whose paths never part
    # differ only by f32 rounding, whose sd alone would set no real bound.
    bias_half = np.maximum(z * diff.std(0, ddof=1) / np.sqrt(n), BIAS_FLOOR * np.abs(other.mean(0)))
    out = {"pixels": n, "relmse_gpu": float(e_g.mean()), "relmse_oracle": float(e_o.mean()),
           "relmse_diff": float(d.mean()), "relmse_half_width": float(half),
           "bias": bias.tolist(), "bias_half_width": bias_half.tolist(), "bias_paired": paired is not None,
           "mean_gpu": gpu.mean(0).tolist(), "mean_oracle": ora.mean(0).tolist()}
    out["ok"] = bool(abs(d.mean()) <= half and (np.abs(bias) <= bias_half + 1e-12).all())
    return out


def render_quad(scene, params, spp, ref_spp, pixel_stride=1, gpu_start=0, ora_start=1 << 22,
                ref_start=1 << 23, oracle_scene=None):
    """G: the GPU's full frame at `spp` (samples from gpu_start); P, O and R:
    the oracle on every `pixel_stride`-th pixel at `spp` over G's samples,
    at `spp` over disjoint samples, and at `ref_spp`. Returns (G, O, R, P)
    on those pixels and the GPU session's stats."""
    import oracle
    from rtcuda import PtSession
    o_s = oracle_scene if oracle_scene is not None else oracle.OracleScene(scene)
    npix = scene.width * scene.height
    pix = np.arange(0, npix, pixel_stride, dtype=np.uint32)
    with PtSession(scene, params) as g:
        g.render_samples(gpu_start, spp)
        gimg = g.image().reshape(-1, 3)[pix]
        st = g.stats()
    paired = o_s.render(params, gpu_start, gpu_start + spp, pixels=pix)[0] / spp
    ora = o_s.render(params, ora_start, ora_start + spp, pixels=pix)[0] / spp
    ref = o_s.render(params, ref_start, ref_start + ref_spp, pixels=pix)[0] / ref_spp
    return gimg, ora, ref, paired, st
