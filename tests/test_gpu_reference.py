"""GPU parity against the reference's own shader compiled for the host.

The checker is oracle/_ref (packages/lib/shader/** compiled as C++ by
oracle/ref/build_ref.sh).  Every product call goes through the C ABI of
libdspbr_cuda.so.
"""
import numpy as np
import pytest

from dspbr import synth
from dspbr.viewport import Bvh, Context, DeviceIbl, DeviceScene, PathtracingViewport
from dspbr import _lib
from oracle import ref_lib
from tests import helpers

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_lib.available("f32"), reason="oracle/_ref not built (needs the reference checkout)")]


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


@pytest.fixture(scope="module")
def small():
    sc = synth.make_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    return sc


@pytest.fixture(scope="module")
def ref32(small):
    r = ref_lib.GlslReference("f32")
    r.set_scene(small.vertices, small.indices, small.materials, small.bvh.nodes, small.bvh.indices)
    r.set_ibl(small.env)
    return r


def _trace_gpu(ctx, ds, rays):
    import ctypes as C
    n = rays.shape[0]
    tri, t, uv = np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros((n, 2), np.float32)
    ctx.check(ctx.lib.dspbr_trace_closest(ctx.h, ds.h, _lib.fptr(np.ascontiguousarray(rays, np.float32)), n,
                                          _lib.iptr(tri), _lib.fptr(t), _lib.fptr(uv)))
    return tri, t, uv


def test_closest_hit_bitexact_small(ctx, small, ref32):
    ds = DeviceScene(ctx, small.vertices, small.indices, small.materials, small.bvh)
    rays = helpers.random_rays(small.vertices, 20000)
    g_tri, g_t, g_uv = _trace_gpu(ctx, ds, rays)
    r_tri, r_t, r_uv = ref32.trace(rays)
    assert (g_tri >= 0).mean() > 0.5
    np.testing.assert_array_equal(g_tri, r_tri)
    np.testing.assert_array_equal(g_t.view(np.uint32), r_t.view(np.uint32))
    np.testing.assert_array_equal(g_uv.view(np.uint32), r_uv.view(np.uint32))


def test_camera_rays_bitexact(ctx, small, ref32):
    v = PathtracingViewport(width=256, height=192)
    v.setCamera(type("Cam", (), {"matrixWorld": small.camera.matrix_world, "fov": small.camera.fov,
                                 "near": small.camera.near})())
    ref32.set_uniforms(ref_lib.uniform_block(small.camera.matrix_world, small.camera.fov, small.camera.near, 256, 192,
                                             1, 8))
    xy, r2 = helpers.camera_rays_ref(ref32, small.camera, 256, 192, 5000)
    out = np.zeros((xy.shape[0], 6), np.float32)
    v.ctx.check(v.ctx.lib.dspbr_camera_rays(v.ctx.h, xy.shape[0], _lib.iptr(xy), _lib.fptr(r2), _lib.fptr(out)))
    ref = ref32.camera_rays(xy, r2, 256, 192)
    np.testing.assert_array_equal(out.view(np.uint32), ref.view(np.uint32))
    v.dispose()


def test_bsdf_against_reference(ctx, small):
    mats = helpers.feature_materials(0)
    ref = ref_lib.GlslReference("f32")
    ref.set_scene(small.vertices, small.indices, mats, small.bvh.nodes, small.bvh.indices)
    ds = DeviceScene(ctx, small.vertices, small.indices, mats, small.bvh)
    hit, wo, rnd = helpers.bsdf_queries(20000, mats.shape[0])
    n = hit.shape[0]
    ev, sm, fl = np.zeros((n, 4), np.float32), np.zeros((n, 10), np.float32), np.zeros(n, np.int32)
    ctx.check(ctx.lib.dspbr_bsdf_query(ctx.h, ds.h, n, _lib.fptr(hit), _lib.fptr(wo), _lib.fptr(rnd), _lib.fptr(ev),
                                       _lib.fptr(sm), _lib.iptr(fl)))
    rev, rsm, rfl = ref.bsdf(hit, wo, rnd)
    np.testing.assert_array_equal(fl, rfl)
    close = np.abs(ev - rev) <= 1e-4 * np.abs(rev) + 1e-6
    frac = close.all(axis=1).mean()
    print("eval/pdf agreement", frac, "max rel", np.max(np.abs(ev - rev) / (np.abs(rev) + 1e-6)))
    assert frac > 0.999
    same_dir = np.all(np.abs(sm[:, 0:3] - rsm[:, 0:3]) <= 1e-4 + 1e-4 * np.abs(rsm[:, 0:3]), axis=1)
    print("sample direction agreement", same_dir.mean())
    assert same_dir.mean() > 0.995
    ok = same_dir[:, None] & ~(np.abs(sm - rsm) <= 1e-3 * np.abs(rsm) + 1e-5)
    print("sample field mismatches where directions agree", ok.sum(axis=0))
    assert ok.any(axis=1).mean() < 0.005


def test_ibl_tables_and_queries(ctx, small, ref32):
    ibl = DeviceIbl(ctx, small.env)
    gt = ibl.tables()
    rt = ref32.ibl_tables()
    for k in ("pdf", "cdf", "yPdf", "yCdf"):
        np.testing.assert_array_equal(gt[k].view(np.uint32), rt[k].view(np.uint32), err_msg=k)
    assert gt["totalSum"] == rt["totalSum"]
    # alias table realises p(x,y) = yPdf[y] * pdf[y,x]
    prob, alias = ibl.alias_table()
    n = prob.size
    mass = prob.astype(np.float64) / n
    np.add.at(mass, alias, (1.0 - prob.astype(np.float64)) / n)
    target = (rt["yPdf"][:, None].astype(np.float64) * rt["pdf"].reshape(small.env.shape[0], -1)).reshape(-1)
    target /= target.sum()
    assert np.max(np.abs(mass - target)) < 1e-6
    # queries in the reference's CDF mode
    rng = np.random.default_rng(4)
    r2 = rng.uniform(size=(5000, 2)).astype(np.float32)
    dirs = helpers.unit(rng, 5000).astype(np.float32)
    p = _lib.default_params()
    p.env_sampling = _lib.ENV_CDF
    ctx.check(ctx.lib.dspbr_set_params(ctx.h, p))
    sdp, pdf, rgb = np.zeros((5000, 4), np.float32), np.zeros(5000, np.float32), np.zeros((5000, 3), np.float32)
    ctx.check(ctx.lib.dspbr_ibl_query(ctx.h, ibl.h, 5000, _lib.fptr(r2), _lib.fptr(dirs), _lib.fptr(sdp),
                                      _lib.fptr(pdf), _lib.fptr(rgb)))
    rsdp, rpdf, rrgb = ref32.ibl(r2, dirs)
    np.testing.assert_allclose(sdp, rsdp, rtol=2e-5, atol=2e-6)
    np.testing.assert_allclose(pdf, rpdf, rtol=2e-5, atol=1e-7)
    np.testing.assert_allclose(rgb, rrgb, rtol=2e-5, atol=2e-6)


def test_image_mwc_matches_reference(small, ref32):
    W, H, F = 96, 96, 8
    v = PathtracingViewport(width=W, height=H, settings={"maxBounces": small.max_bounces, "envSampling": "cdf"})
    v.setScene(small)
    v.setIBL(small.env)
    v.setCamera(type("Cam", (), {"matrixWorld": small.camera.matrix_world, "fov": small.camera.fov,
                                 "near": small.camera.near})())
    v.start(F)
    img = v.readAccumulation()
    acc = np.zeros((H, W, 4), np.float32)
    for f in range(1, F + 1):
        ref32.set_uniforms(ref_lib.uniform_block(small.camera.matrix_world, small.camera.fov, small.camera.near, W, H,
                                                 f, small.max_bounces))
        ref32.render(W, H, acc)
    diff = np.abs(img[..., :3] - acc[..., :3])
    close = np.all(diff <= 1e-3 * np.abs(acc[..., :3]) + 1e-4, axis=-1)
    print("pixels matching the reference path-for-path:", close.mean(), "mean abs diff", diff.mean())
    assert close.mean() > 0.95
    assert diff.mean() < 0.01 * acc[..., :3].mean()
    v.dispose()
