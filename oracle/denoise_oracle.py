"""Test infrastructure only (the checker, never the product): an f64 numpy
restatement of the reference's AOV-guided denoiser,
src/output/denoise.rs:28-139 (edge-avoiding a-trous wavelet filter after
Dammertz et al. 2010). Pinned by the reference's own test of that file
(denoise_reduces_noise_preserves_edges), restated in tests/test_film_cpu.py.

The film is a dict of (H, W, k) arrays: diffuse, specular, albedo, normal,
depth (k = 1 or more, first channel used) and id (first channel used)."""
import numpy as np

KERNEL = np.array([1.0 / 16.0, 1.0 / 4.0, 3.0 / 8.0, 1.0 / 4.0, 1.0 / 16.0])  # denoise.rs:18
ITERATIONS = 5                                                              # denoise.rs:19


def _lum(c):
    return 0.2126 * c[..., 0] + 0.7152 * c[..., 1] + 0.0722 * c[..., 2]     # denoise.rs:21-23


def denoise(film):
    diffuse = np.asarray(film["diffuse"], np.float64)[..., :3]
    specular = np.asarray(film["specular"], np.float64)[..., :3]
    albedo = np.asarray(film["albedo"], np.float64)[..., :3]
    normal = np.asarray(film["normal"], np.float64)[..., :3]
    depth = np.asarray(film["depth"], np.float64)[..., 0]
    oid = np.asarray(film["id"], np.float64)[..., 0]
    h, w = diffuse.shape[:2]
    if h == 0 or w == 0:
        return np.asarray(film["beauty"], np.float64)
    a = np.maximum(albedo, 5e-2)
    illum = diffuse / a                                                     # denoise.rs:36-52
    pos = np.sort(depth[depth > 0.0])                                       # denoise.rs:55-63
    depth_scale = max(pos[len(pos) // 2] if len(pos) else 1.0, 1e-3)
    sigma_c = 8.0
    for it in range(ITERATIONS):                                            # denoise.rs:67-114
        step = 1 << it
        src = illum
        s = np.zeros_like(src)
        ws = np.zeros((h, w))
        for kj in range(5):
            dy = (kj - 2) * step
            for ki in range(5):
                dx = (ki - 2) * step
                # neighbour (y + dy, x + dx), valid where inside the image
                ys0, ys1 = max(0, -dy), min(h, h - dy)
                xs0, xs1 = max(0, -dx), min(w, w - dx)
                if ys0 >= ys1 or xs0 >= xs1:
                    continue
                c0 = src[ys0:ys1, xs0:xs1]
                cn = src[ys0 + dy:ys1 + dy, xs0 + dx:xs1 + dx]
                wgt = KERNEL[kj] * KERNEL[ki]
                dc = _lum(cn - c0)
                wgt = wgt * np.exp(-(dc * dc) / (sigma_c * sigma_c))
                nd = np.maximum(np.einsum("ijk,ijk->ij", normal[ys0 + dy:ys1 + dy, xs0 + dx:xs1 + dx],
                                          normal[ys0:ys1, xs0:xs1]), 0.0)
                wgt = wgt * nd ** 32
                dd = (depth[ys0 + dy:ys1 + dy, xs0 + dx:xs1 + dx] - depth[ys0:ys1, xs0:xs1]) / depth_scale
                wgt = wgt * np.exp(-(dd * dd) / 0.02)
                wgt = np.where(np.abs(oid[ys0 + dy:ys1 + dy, xs0 + dx:xs1 + dx] - oid[ys0:ys1, xs0:xs1]) > 0.5,
                               0.0, wgt)
                s[ys0:ys1, xs0:xs1] += cn * wgt[..., None]
                ws[ys0:ys1, xs0:xs1] += wgt
        illum = np.where(ws[..., None] > 1e-9, s / np.maximum(ws, 1e-300)[..., None], src)
        sigma_c *= 0.5
    return illum * a + specular                                             # denoise.rs:117-134
