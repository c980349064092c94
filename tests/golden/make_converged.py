#!/usr/bin/env python3
"""Generates tests/golden/converged_small_f64.npz: the converged-image fixture.

The small configuration's scene (Cornell-style box, two boxes, icosphere, glass
sphere; 256x128 environment with a sun lobe) rendered at 128x128 with 8
bounces by the reference's own fragment shader compiled for the host in FP64
(oracle/ref/build_ref.sh, GLSL_REAL=double): renderer.frag:146-157 over
integrator/misptdl.glsl:34-93, the reference's MWC RNG (rng.glsl) and its
two-level CDF environment sampling (lighting.glsl:24-42).  4096 progressive
frames, one sample per pixel each.  Stored per pixel: the mean and the sample
variance of the RGB radiance over the 4096 samples (float32), and the inputs
that define the scene, so that the fixture stands alone.

Run from the repository root where the reference checkout is available:
    python tests/golden/make_converged.py
(about 3 minutes on 8 host cores).
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "dspbr-pt_b200"))

from dspbr import synth  # noqa: E402
from dspbr.viewport import Bvh  # noqa: E402
from oracle import oracle_lib, ref_lib  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "converged_small_f64.npz")
W, H, SPP, BOUNCES = 128, 128, 4096, 8


def main():
    sc = synth.make_small(0)
    bvh = Bvh.build(sc.vertices, sc.indices, 20)
    ref = ref_lib.GlslReference("f64")
    ref.set_scene(sc.vertices, sc.indices, sc.materials, bvh.nodes, bvh.indices)
    ref.set_ibl(sc.env)
    xy = oracle_lib.all_pixels(W, H)
    s1 = np.zeros((H * W, 3), np.float64)
    s2 = np.zeros((H * W, 3), np.float64)
    rays = 0
    t0 = time.time()
    for f in range(1, SPP + 1):
        ref.set_uniforms(ref_lib.uniform_block(sc.camera.matrix_world, sc.camera.fov, sc.camera.near, W, H, f,
                                               BOUNCES))
        out, r = ref.render_pixels(xy, W, H)
        # render_pixels returns the running mean over a zero previous frame,
        # contribution / frame (renderer.frag:153-154): undo the division
        c = out[:, :3].astype(np.float64) * f
        s1 += c
        s2 += c * c
        rays += r
    mean = s1 / SPP
    var = np.maximum(s2 / SPP - mean * mean, 0.0) * (SPP / (SPP - 1.0))
    np.savez_compressed(OUT, mean=mean.reshape(H, W, 3).astype(np.float32),
                        var=var.reshape(H, W, 3).astype(np.float32),
                        whsb=np.array([W, H, SPP, BOUNCES], np.int32),
                        vertices=sc.vertices, indices=sc.indices, materials=sc.materials, env=sc.env,
                        cam_matrix=sc.camera.matrix_world,
                        cam_fov_near=np.array([sc.camera.fov, sc.camera.near], np.float64))
    print(f"wrote {OUT}: {SPP} spp at {W}x{H}, {rays / 1e6:.0f} M rays in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
