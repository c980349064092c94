"""Converged-image gate: the CUDA path at 4096 samples per pixel against the
FP64 oracle at 4096 samples per pixel.

The fixture (tests/golden/converged_small_f64.npz, made by make_converged.py)
holds the per-pixel mean and sample variance of the reference's own fragment
shader compiled for the host in FP64 (renderer.frag:146-157 over
integrator/misptdl.glsl:34-93), with the reference's MWC RNG (rng.glsl:5-29)
and its two-level CDF environment sampling (lighting.glsl:24-42).  The GPU
renders the same scene with PCG32 streams per pixel sample and the alias-table
environment sampler: an independent sample stream of the same estimator, so
the difference of the two means is noise of known variance unless the
estimators differ.  The GPU's own per-pixel variance comes from 64 batches of
64 samples (independent seeds): the standard error of the difference is
sqrt((var_oracle + var_gpu) / N) with N = 4096 on both sides.  Using the
oracle's variance alone skews z: where the oracle drew a rare bright sample
(a caustic through the glass sphere, the sun lobe) its variance is large, and
where it drew none its variance is small while the GPU's mean may hold one.

Bars (per pixel and colour channel):
  * |z| < 4 for at least 99.9% of the pixel channels, and |z| < 8 for all;
  * the mean z over the image within +-0.05 (no global bias);
  * RMSE(GPU - oracle) at most 1.1 x the RMSE that noise alone gives,
    sqrt(mean((var_oracle + var_gpu) / N)).
Measured on a B200 (both traversals; the same 49152 channels): |z| < 4 on
99.988%, max |z| 4.65, mean z +0.013, RMSE 4.34e-3 against 4.39e-3 from
noise alone (ratio 0.99).  The CPU restatement (oracle/dspbr_oracle.cpp)
run through the same procedure draws the same PCG samples and gives the same
figures to the printed digits.
"""
import os

import numpy as np
import pytest

from dspbr import synth
from dspbr.viewport import PathtracingCamera, PathtracingViewport

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "converged_small_f64.npz")

Z_BOUND, Z_PASS_FRACTION, Z_MAX = 4.0, 0.999, 8.0
MEAN_Z_BOUND = 0.05
RMSE_NOISE_FACTOR = 1.1
BATCHES = 64


def render_converged(g, traversal):
    """Per-pixel mean and sample variance of N samples rendered as BATCHES
    batches of N / BATCHES samples with independent PCG seeds."""
    W, H, N, B = (int(x) for x in g["whsb"])
    fov, near = (float(x) for x in g["cam_fov_near"])
    cam = synth.Camera(g["cam_matrix"], fov, near)
    sc = synth.Scene("converged", g["vertices"], g["indices"], g["materials"], cam, env=g["env"])
    v = PathtracingViewport(width=W, height=H, settings={"maxBounces": B, "rng": "pcg", "seed": 20241,
                                                         "envSampling": "alias", "traversal": traversal})
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(PathtracingCamera(cam.matrix_world, fov, near))
    per = N // BATCHES
    means = np.zeros((BATCHES, H, W, 3))
    for k in range(BATCHES):
        v.setSettings({"seed": 20241 + 7919 * k})  # resets the accumulation
        v.start(per)
        means[k] = v.readAccumulation()[..., :3]
        d = v.diagnostics
        assert d["sample_count"] == per and d["traversal_aborted"] == 0
    v.dispose()
    assert np.isfinite(means).all()
    # the variance of one sample from the spread of the batch means
    return means.mean(0), means.var(0, ddof=1) * per, N


@pytest.mark.parametrize("traversal", ["wide", "reference"])
def test_converged_image_matches_fp64_oracle_at_4096_spp(traversal):
    g = dict(np.load(FIXTURE))
    img, var_g, n = render_converged(g, traversal)
    mean = g["mean"].astype(np.float64)
    var_o = g["var"].astype(np.float64)
    se = np.sqrt((var_o + var_g) / n + (1e-6 * np.abs(mean)) ** 2)
    z = (img - mean) / se
    rmse = float(np.sqrt(((img - mean) ** 2).mean()))
    rmse_noise = float(np.sqrt(((var_o + var_g) / n).mean()))
    frac = float((np.abs(z) < Z_BOUND).mean())
    worst = np.argsort(np.abs(z).ravel())[-3:]
    print(f"{traversal}: |z|<{Z_BOUND} on {frac:.5f} of pixel channels, max |z| {np.abs(z).max():.2f}, "
          f"mean z {z.mean():+.4f}; RMSE {rmse:.3e} (noise alone {rmse_noise:.3e}, ratio {rmse / rmse_noise:.3f}); "
          f"image mean {img.mean():.5f} vs {mean.mean():.5f}; largest |z| at gpu/oracle "
          f"{[(round(float(img.ravel()[i]), 4), round(float(mean.ravel()[i]), 4)) for i in worst]}")
    assert frac >= Z_PASS_FRACTION
    assert np.abs(z).max() < Z_MAX
    assert abs(z.mean()) < MEAN_Z_BOUND
    assert rmse <= RMSE_NOISE_FACTOR * rmse_noise
