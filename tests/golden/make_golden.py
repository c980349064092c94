#!/usr/bin/env python3
"""Generates the golden vectors in this directory from the reference itself.

The reference has no tests or known-answer vectors of its own; these fixtures
are outputs of its own fragment shader (packages/lib/shader/**), compiled for
the host by oracle/ref/build_ref.sh and driven by oracle/ref/ref_harness.cpp.
Inputs are stored beside the outputs so that the fixtures stand alone.

Run from the repository root where the reference checkout is available:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "dspbr-pt_b200"))

from dspbr import synth  # noqa: E402
from dspbr.viewport import Bvh  # noqa: E402
from oracle import ref_lib  # noqa: E402
from tests import helpers  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    sc = synth.make_small(0)
    bvh = Bvh.build(sc.vertices, sc.indices, 20)
    mats = helpers.feature_materials(0)
    env = synth.env_sun(64, 32, 0.3, sc.meta["sun"], 500.0, 6.0)
    r32, r64 = ref_lib.GlslReference("f32"), ref_lib.GlslReference("f64")
    for r in (r32, r64):
        r.set_scene(sc.vertices, sc.indices, mats, bvh.nodes, bvh.indices)
        r.set_ibl(env)
    g = {"vertices": sc.vertices, "indices": sc.indices, "materials": mats, "bvh_nodes": bvh.nodes,
         "bvh_indices": bvh.indices, "env": env}
    # closest hit / occlusion (bvh.glsl:149-229)
    rays = helpers.random_rays(sc.vertices, 2000, seed=11)
    g["rays"] = rays
    g["hit_tri"], g["hit_t"], g["hit_uv"] = r32.trace(rays)
    g["occluded"] = r32.occluded(rays)
    # camera rays (renderer.frag:129-142) and RNG (rng.glsl)
    W, H = 64, 48
    r32.set_uniforms(ref_lib.uniform_block(sc.camera.matrix_world, sc.camera.fov, sc.camera.near, W, H, 1, 8))
    xy, r2 = helpers.camera_rays_ref(r32, sc.camera, W, H, 500, seed=12)
    g["cam_matrix"] = sc.camera.matrix_world
    g["cam_fov_near_wh"] = np.array([sc.camera.fov, sc.camera.near, W, H], np.float64)
    g["cam_xy"], g["cam_r2"] = xy, r2
    g["cam_rays"] = r32.camera_rays(xy, r2, W, H)
    g["rng_args"] = np.array([[5, 9, 16], [0, 0, 8], [511, 511, 2048]], np.int32)
    g["rng_out"] = np.stack([r32.rng(int(x), int(y), int(s), 32) for x, y, s in g["rng_args"]])
    # BSDF through configure_gltf_material + pbr* (material.glsl, material_kernel.glsl)
    hit, wo, rnd = helpers.bsdf_queries(2000, mats.shape[0], seed=13)
    g["bsdf_hit"], g["bsdf_wo"], g["bsdf_rnd"] = hit, wo, rnd
    g["bsdf_eval32"], g["bsdf_sample32"], g["bsdf_flags"] = r32.bsdf(hit, wo, rnd)
    g["bsdf_eval64"], g["bsdf_sample64"], _ = r64.bsdf(hit, wo, rnd)
    # IBL tables (renderer.ts:777-838) and queries (lighting.glsl:24-98)
    t = r32.ibl_tables()
    for k in ("pdf", "cdf", "yPdf", "yCdf"):
        g["ibl_" + k] = t[k]
    g["ibl_totalSum"] = np.array([t["totalSum"]])
    rng = np.random.default_rng(14)
    ir2 = rng.uniform(size=(1000, 2)).astype(np.float32)
    idirs = helpers.unit(rng, 1000).astype(np.float32)
    g["ibl_r2"], g["ibl_dirs"] = ir2, idirs
    g["ibl_sample"], g["ibl_pdf_at"], g["ibl_rgb_at"] = r32.ibl(ir2, idirs)
    # a small progressive image of the small scene (renderer.frag:146-157)
    r32.set_scene(sc.vertices, sc.indices, sc.materials, bvh.nodes, bvh.indices)
    r32.set_ibl(sc.env)
    W, H, F = 32, 32, 4
    acc = np.zeros((H, W, 4), np.float32)
    for f in range(1, F + 1):
        r32.set_uniforms(ref_lib.uniform_block(sc.camera.matrix_world, sc.camera.fov, sc.camera.near, W, H, f, 8))
        r32.render(W, H, acc)
    g["image_scene_materials"] = sc.materials
    g["image_env"] = sc.env
    g["image_whf"] = np.array([W, H, F], np.int32)
    g["image"] = acc
    np.savez_compressed(os.path.join(OUT, "reference_small.npz"), **g)
    print("wrote", os.path.join(OUT, "reference_small.npz"))


if __name__ == "__main__":
    main()
