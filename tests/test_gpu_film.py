"""The AOV film and the denoiser on the GPU (csrc/film.cu) against the f64
oracle restatement of src/output/denoise.rs (oracle/denoise_oracle.py) and
the reference's own denoise test, and the device film decode against the
host decode of render_pt_film (renderer.rs:180-217)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import denoise_oracle  # noqa: E402  (the checker)

from rtcuda import PtSession, abi, scenes  # noqa: E402
from rtcuda.backend import decode_film, denoise_film, film_array  # noqa: E402
from test_film_cpu import check_reference_denoise_properties, noisy_halves_film  # noqa: E402

pytestmark = pytest.mark.gpu


def test_reference_denoise_test_on_the_gpu():
    film = noisy_halves_film()
    out = denoise_film(film)
    check_reference_denoise_properties(film, out)
    np.testing.assert_allclose(out, denoise_oracle.denoise(film), atol=2e-4)


def test_rendered_film_and_denoise_match_the_oracle():
    s = scenes.cornell_box(96, 72)
    spp = 8
    with PtSession(s, abi.make_params(max_depth=8, aovs=True)) as g:
        g.render_samples(0, spp)
        film = g.film()
        host = decode_film(g.image(), g.aux(), spp)
        den = g.denoise()
    for k in ("beauty", "diffuse", "specular", "albedo", "normal", "depth", "id"):
        np.testing.assert_allclose(film[k], np.asarray(host[k], np.float32), rtol=1e-5, atol=1e-6, err_msg=k)
    ref = denoise_oracle.denoise({k: v.astype(np.float64) for k, v in film.items()})
    np.testing.assert_allclose(den, ref, rtol=2e-3, atol=2e-3)
    # Same film through the session-free entry point: identical result.
    np.testing.assert_array_equal(denoise_film(film_array(film)), den)
    # The filter removes pixel-scale noise (energy above a 3x3 box blur)
    # away from the light source, whose bright edge pixels it keeps apart.
    def shift_sum(a):
        return sum(np.roll(np.roll(a, dy, 0), dx, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1))
    bright = film["beauty"].max(-1) > 1.0
    keep = ~(shift_sum(shift_sum(bright.astype(np.float32))) > 0)
    keep[:2], keep[-2:], keep[:, :2], keep[:, -2:] = False, False, False, False
    hf = lambda img: float(((img - shift_sum(img) / 9.0) ** 2).sum(-1)[keep].mean())
    assert keep.sum() > 0.5 * keep.size
    assert hf(den) < 0.5 * hf(film["beauty"]), (hf(den), hf(film["beauty"]))
    assert np.isfinite(den).all() and den.min() >= 0.0


def test_film_needs_aovs():
    s = scenes.cornell_box(8, 8)
    with PtSession(s, abi.make_params(max_depth=4)) as g:
        g.render_samples(0, 1)
        with pytest.raises(Exception, match="AOVs"):
            g.denoise()
