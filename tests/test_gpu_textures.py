"""Material textures on the GPU (dspbr_scene_set_textures): RGBA8 texture
arrays sampled LINEAR + REPEAT through TexInfo records, every texture slot of
configure_gltf_material (material.glsl:5-110), against golden vectors made by
the reference's own shaders with the same textures."""
import numpy as np
import pytest

from dspbr import _lib, synth
from dspbr.viewport import Bvh, Context, DeviceScene, PathtracingViewport
from tests import helpers
from tests.test_gpu_parity import (BSDF_ATOL, BSDF_MIN_FRACTION, BSDF_RTOL, SAMPLE_MIN_FRACTION, _bsdf_agreement,
                                   bsdf_gpu, ref_params)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    return helpers.load_golden()


def test_textured_bsdf_matches_reference_golden(g):
    import ctypes as C
    ctx = Context(0)
    ctx.check(ctx.lib.dspbr_set_params(ctx.h, C.byref(ref_params())))
    bvh = Bvh(g["bvh_nodes"], g["bvh_indices"], 0, g["indices"].size // 3)
    ds = DeviceScene(ctx, g["vertices"], g["indices"], g["tex_materials"], bvh)
    hit, wo, rnd = g["tex_bsdf_hit"], g["tex_bsdf_wo"], g["tex_bsdf_rnd"]
    with pytest.raises(_lib.DspbrError):  # textures not set yet
        bsdf_gpu(ctx, ds, hit, wo, rnd)
    ds.set_textures(g["tex_infos"], [g["tex_array0"], g["tex_array1"]])
    ev, sm, fl = bsdf_gpu(ctx, ds, hit, wo, rnd)
    np.testing.assert_array_equal(fl, g["tex_bsdf_flags"])
    e, d, smp = _bsdf_agreement(ev, sm, g["tex_bsdf_eval32"], g["tex_bsdf_sample32"])
    print("textured: eval/pdf agree", e, "same direction", d, "samples agree", smp)
    assert e >= BSDF_MIN_FRACTION and smp >= SAMPLE_MIN_FRACTION
    ds.close()
    ctx.close()


def test_set_textures_validates_ids(g):
    ctx = Context(0)
    bvh = Bvh(g["bvh_nodes"], g["bvh_indices"], 0, g["indices"].size // 3)
    ds = DeviceScene(ctx, g["vertices"], g["indices"], g["tex_materials"], bvh)
    with pytest.raises(_lib.DspbrError):  # the materials use ids up to 8
        ds.set_textures(g["tex_infos"][:3], [g["tex_array0"]])
    ds.close()
    ctx.close()


@pytest.mark.parametrize("traversal", ["reference", "wide"])
def test_textured_image_matches_golden_path_for_path(g, traversal):
    sc = synth.make_textured_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    W, H, F = (int(x) for x in g["tex_image_whf"])
    v = PathtracingViewport(width=W, height=H, settings={"maxBounces": 8, "envSampling": "cdf",
                                                        "traversal": traversal})
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(helpers.camera_of(sc))
    v.start(F)
    img = v.readAccumulation()
    v.dispose()
    ref = g["tex_image"]
    close = helpers.close_mask(img[..., :3], ref[..., :3], 1e-3, 1e-4).all(-1)
    print("textured pixels equal to the reference path for path:", close.mean())
    assert close.mean() >= 0.99  # measured 0.9941 (reference traversal), 0.9922 (wide)
    assert np.abs(img - ref).mean() < 0.01 * ref[..., :3].mean()


def test_server_mixes_textured_and_untextured_requests():
    from dspbr.server import Server
    from dspbr.viewport import DeviceIbl
    ctx = Context(0)
    tex, plain = synth.make_textured_small(0), synth.make_small(0)
    scenes, ibls = [], []
    for sc in (tex, plain):
        sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
        ds = DeviceScene(ctx, sc.vertices, sc.indices, sc.materials, sc.bvh)
        if getattr(sc, "tex_infos", None) is not None:
            ds.set_textures(sc.tex_infos, sc.tex_arrays)
        scenes.append(ds)
        ibls.append(DeviceIbl(ctx, sc.env))
    reqs = [(0, 48, 40, 3), (1, 40, 32, 4), (0, 17, 9, 2)]

    def submit(srv, r):
        k, w, h, spp = r
        sc = (tex, plain)[k]
        return srv.submit(scenes[k], ibls[k], helpers.camera_of(sc), w, h, spp, {"maxBounces": 6})

    alone = []
    for r in reqs:
        srv = Server(ctx, path_pool=1 << 16)
        img, info = srv.wait(submit(srv, r))
        srv.close()
        assert info["state"] == "done"
        alone.append(img.copy())
    srv = Server(ctx, path_pool=3000)
    ids = [submit(srv, r) for r in reqs]
    mix = [srv.wait(i, timeout_ms=120000)[0].copy() for i in ids]
    srv.close()
    for a, m in zip(alone, mix):
        np.testing.assert_allclose(m, a, rtol=1e-6, atol=1e-7)
    assert all(np.isfinite(a).all() and a[..., :3].max() > 0 for a in alone)
    for o in scenes + ibls:
        o.close()
    ctx.close()
