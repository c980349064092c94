#!/usr/bin/env python3
"""Generates the golden vectors in this directory from the reference itself.

The reference has no tests or known-answer vectors of its own; these fixtures
are outputs of its own fragment shader (packages/lib/shader/**), compiled for
the host by oracle/ref/build_ref.sh and driven by oracle/ref/ref_harness.cpp.
Inputs are stored beside the outputs so that the fixtures stand alone.

Run from the repository root where the reference checkout is available:
    python tests/golden/make_golden.py
"""
import hashlib
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


def display_test_image(w, h):
    """Seeded HDR image: log-uniform radiance noise, a bright disc with a hard
    edge, diagonal stripes and a zero / negative-free alpha ramp."""
    rng = np.random.default_rng(15)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    img = np.exp(rng.uniform(np.log(1e-4), np.log(20.0), (h, w, 3))).astype(np.float32)
    disc = (x - w * 0.6) ** 2 + (y - h * 0.4) ** 2 < (0.25 * h) ** 2
    img[disc] = [8.0, 6.0, 3.0]
    stripes = ((x + y) // 3) % 2 == 0
    img[stripes & ~disc] *= 0.05
    img[:, :2] = 0.0
    alpha = (x / (w - 1)).astype(np.float32)[..., None]
    return np.ascontiguousarray(np.concatenate([img, alpha], -1), np.float32)


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
    # display epilogue (tonemap.frag, fxaa.frag) over an HDR test image with
    # hard edges and a dark-to-bright ramp, and over the rendered image
    hdr = display_test_image(48, 40)
    g["display_hdr"] = hdr
    modes = [-1, 0, 1, 2, 3, 4]
    g["display_modes"] = np.array(modes, np.int32)
    for gamma in (0, 1):
        g[f"display_tonemap_g{gamma}"] = np.stack([r32.tonemap(hdr, 1.7, gamma, m) for m in modes])
    tm = r32.tonemap(hdr, 1.0, 1, 3)
    g["display_fxaa_in"] = tm
    g["display_fxaa"] = r32.fxaa(tm)
    g["display_image_aces_fxaa"] = r32.fxaa(r32.tonemap(acc, 1.0, 1, 3))
    # material textures (scene_data_webgl2.ts:233-363, material.glsl:5-110):
    # BSDF queries over textured feature materials, and a textured image
    tinfos, tarrays = synth.texture_set(3)
    tmats = synth.texture_materials(mats, 4)
    g["tex_infos"] = tinfos
    g["tex_array0"], g["tex_array1"] = tarrays
    g["tex_materials"] = tmats
    for r in (r32, r64):
        r.set_scene(sc.vertices, sc.indices, tmats, bvh.nodes, bvh.indices)
        r.set_textures(tinfos, tarrays)
    thit, two, trnd = helpers.bsdf_queries(3000, tmats.shape[0], seed=16)
    thit[:, 13:15] = np.random.default_rng(17).uniform(-1.5, 2.5, size=(3000, 2))  # wrap-around uvs
    g["tex_bsdf_hit"], g["tex_bsdf_wo"], g["tex_bsdf_rnd"] = thit, two, trnd
    g["tex_bsdf_eval32"], g["tex_bsdf_sample32"], g["tex_bsdf_flags"] = r32.bsdf(thit, two, trnd)
    g["tex_bsdf_eval64"], g["tex_bsdf_sample64"], _ = r64.bsdf(thit, two, trnd)
    ts = synth.make_textured_small(0)
    tbvh = Bvh.build(ts.vertices, ts.indices, 20)
    r32.set_scene(ts.vertices, ts.indices, ts.materials, tbvh.nodes, tbvh.indices)
    r32.set_textures(ts.tex_infos, ts.tex_arrays)
    r32.set_ibl(ts.env)
    W, H, F = 32, 32, 4
    acc = np.zeros((H, W, 4), np.float32)
    for f in range(1, F + 1):
        r32.set_uniforms(ref_lib.uniform_block(ts.camera.matrix_world, ts.camera.fov, ts.camera.near, W, H, f, 8))
        assert r32.render(W, H, acc) is not None
    g["tex_image"] = acc
    g["tex_image_whf"] = np.array([W, H, F], np.int32)
    # the point light (lighting.glsl:2-22, misptdl.glsl:24-30): the small scene
    # with a light under the ceiling, as the first scene light sets it
    # (renderer.ts:424-430)
    ps = synth.make_small(0)
    pbvh = Bvh.build(ps.vertices, ps.indices, 20)
    r32.set_scene(ps.vertices, ps.indices, ps.materials, pbvh.nodes, pbvh.indices)
    r32.set_ibl(ps.env)
    light = ((0.2, 1.7, 0.3), (6.0, 5.0, 4.0))
    W, H, F = 32, 32, 4
    acc = np.zeros((H, W, 4), np.float32)
    for f in range(1, F + 1):
        r32.set_uniforms(ref_lib.uniform_block(ps.camera.matrix_world, ps.camera.fov, ps.camera.near, W, H, f, 8,
                                               point_light=light))
        assert r32.render(W, H, acc) is not None
    g["pl_image"] = acc
    g["pl_light"] = np.array(light, np.float32)
    g["pl_image_whf"] = np.array([W, H, F], np.int32)
    # a glTF asset packed by dspbr.gltf (scene_loader.ts), rendered by the
    # reference shaders with its textures
    from dspbr.gltf_writer import sample_camera, sample_scene
    from dspbr import gltf
    gs = gltf.load_gltf(sample_scene().glb_bytes())
    cam = sample_camera()
    gbvh = Bvh.build(gs.vertices, gs.indices, 20)
    r32.set_scene(gs.vertices, gs.indices, gs.materials, gbvh.nodes, gbvh.indices)
    r32.set_textures(gs.tex_infos, gs.tex_arrays)
    r32.set_ibl(ps.env)
    W, H, F = 48, 36, 4
    acc = np.zeros((H, W, 4), np.float32)
    for f in range(1, F + 1):
        r32.set_uniforms(ref_lib.uniform_block(cam.matrix_world, cam.fov, cam.near, W, H, f, 8))
        assert r32.render(W, H, acc) is not None
    g["gltf_image"] = acc
    g["gltf_image_whf"] = np.array([W, H, F], np.int32)
    # the divergence configuration's materials (transmission, volume absorption,
    # dispersion, iridescence) at 32 bounces, path for path
    dv = synth.make_divergence_small(0)
    dbvh = Bvh.build(dv.vertices, dv.indices, 20)
    r32.set_scene(dv.vertices, dv.indices, dv.materials, dbvh.nodes, dbvh.indices)
    r32.set_textures(gltf.DEFAULT_TEX_INFO.reshape(1, 8), [])
    r32.set_ibl(dv.env)
    W, H, F = dv.width, dv.height, 4
    acc = np.zeros((H, W, 4), np.float32)
    for f in range(1, F + 1):
        r32.set_uniforms(ref_lib.uniform_block(dv.camera.matrix_world, dv.camera.fov, dv.camera.near, W, H, f, 32))
        assert r32.render(W, H, acc) is not None
    g["div_image"] = acc
    g["div_image_whf"] = np.array([W, H, F], np.int32)
    g["gltf_vertices_sha"] = np.frombuffer(hashlib.sha256(gs.vertices.tobytes() + gs.indices.tobytes() +
                                                          gs.materials.tobytes() + gs.tex_infos.tobytes()).digest(),
                                           np.uint8)
    np.savez_compressed(os.path.join(OUT, "reference_small.npz"), **g)
    print("wrote", os.path.join(OUT, "reference_small.npz"))


if __name__ == "__main__":
    main()
