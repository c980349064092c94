"""Converged-image gate: the CUDA path at 4096 samples per pixel against the
FP64 oracle at 4096 samples per pixel.

The fixture (tests/golden/converged_small_f64.npz, made by make_converged.py)
holds the per-pixel mean and sample variance of the reference's own fragment
shader compiled for the host in FP64 (renderer.frag:146-157 over
integrator/misptdl.glsl:34-93), with the reference's MWC RNG (rng.glsl:5-29)
and its two-level CDF environment sampling (lighting.glsl:24-42).  The GPU
renders the same scene with PCG32 streams per pixel sample and the alias-table
environment sampler: an independent sample stream of the same estimator, so
the difference of the two means is pure noise of known variance unless the
estimators differ.

Bars (per pixel and channel; N = 4096 on both sides; the standard error of
the difference is sqrt(2 var / N) with the oracle's per-pixel variance):
  * |z| < 4 for at least 99.9% of the pixel channels, and |z| < 8 for all;
  * the mean z over the image within +-0.03 (no global bias);
  * RMSE(GPU - oracle) at most 1.2 x the RMSE that noise alone gives,
    sqrt(mean(2 var / N)), and below 1e-3 absolute.
"""
import os

import numpy as np
import pytest

from dspbr import synth
from dspbr.viewport import PathtracingCamera, PathtracingViewport

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "converged_small_f64.npz")

Z_BOUND, Z_PASS_FRACTION, Z_MAX = 4.0, 0.999, 8.0
MEAN_Z_BOUND = 0.03
RMSE_NOISE_FACTOR, RMSE_ABS = 1.2, 1e-3


def render_converged(g, traversal):
    W, H, N, B = (int(x) for x in g["whsb"])
    fov, near = (float(x) for x in g["cam_fov_near"])
    cam = synth.Camera(g["cam_matrix"], fov, near)
    sc = synth.Scene("converged", g["vertices"], g["indices"], g["materials"], cam, env=g["env"])
    v = PathtracingViewport(width=W, height=H, settings={"maxBounces": B, "rng": "pcg", "seed": 20241,
                                                         "envSampling": "alias", "traversal": traversal})
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(PathtracingCamera(cam.matrix_world, fov, near))
    v.start(N)
    img = v.readAccumulation()
    d = v.diagnostics
    v.dispose()
    assert d["sample_count"] == N and d["rays_primary"] == W * H * N and d["traversal_aborted"] == 0
    return img[..., :3].astype(np.float64), N


@pytest.mark.parametrize("traversal", ["wide", "reference"])
def test_converged_image_matches_fp64_oracle_at_4096_spp(traversal):
    g = dict(np.load(FIXTURE))
    img, n = render_converged(g, traversal)
    mean = g["mean"].astype(np.float64)
    var = g["var"].astype(np.float64)
    se = np.sqrt(2.0 * var / n + (1e-6 * np.abs(mean)) ** 2)
    z = (img - mean) / se
    rmse = float(np.sqrt(((img - mean) ** 2).mean()))
    rmse_noise = float(np.sqrt((2.0 * var / n).mean()))
    frac = float((np.abs(z) < Z_BOUND).mean())
    print(f"{traversal}: |z|<{Z_BOUND} on {frac:.5f} of pixel channels, max |z| {np.abs(z).max():.2f}, "
          f"mean z {z.mean():+.4f}; RMSE {rmse:.3e} (noise alone {rmse_noise:.3e}, ratio {rmse / rmse_noise:.3f}); "
          f"image mean {img.mean():.5f} vs {mean.mean():.5f}")
    assert np.isfinite(img).all()
    assert frac >= Z_PASS_FRACTION
    assert np.abs(z).max() < Z_MAX
    assert abs(z.mean()) < MEAN_Z_BOUND
    assert rmse <= RMSE_NOISE_FACTOR * rmse_noise and rmse < RMSE_ABS
