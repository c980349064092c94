"""The compressed 8-wide BVH (dspbr_set_wide_bvh(ctx, 8); device.cuh cw8_step,
bvh_gpu.cu k_cw8_level) against the reference's binary traversal
(bvh.glsl:149-229) on the same scenes.

Bars: hit/miss and the closest t bit for bit on random and camera rays; the
triangle may differ only where two triangles hit at exactly that t.  On the
golden scene (boxes standing on the floor: coplanar faces) the closest t may
also differ by a tie within rounding, t within 1e-6 relative, where the
triangle found here is the brute-force closest one: the reference's own
result in such a tie depends on which face its traversal meets first.
"""
import numpy as np
import pytest

from dspbr import _lib, synth
from dspbr.viewport import Bvh, Context, DeviceScene, PathtracingCamera, PathtracingViewport
from oracle import oracle_lib
from tests import helpers
from tests.test_gpu_parity import set_traversal, trace_gpu
from tests.test_gpu_refit import _deform

pytestmark = pytest.mark.gpu

TIE_REL = 1e-6


def wide8_context(builder=None):
    c = Context(0)
    set_traversal(c, _lib.TRAVERSAL_WIDE)
    c.set_wide_bvh(8)
    if builder:
        c.set_bvh_builder(builder)
    return c


@pytest.fixture(scope="module")
def ctx_ref():
    c = Context(0)
    set_traversal(c, _lib.TRAVERSAL_REFERENCE)
    return c


@pytest.fixture(scope="module")
def ctx8():
    return wide8_context()


def check_same_t(tri, t, rtri, rt):
    np.testing.assert_array_equal(tri >= 0, rtri >= 0)
    np.testing.assert_array_equal(t.view(np.uint32), rt.view(np.uint32))
    assert (tri != rtri).mean() < 1e-3  # exact t-ties only


@pytest.mark.parametrize("ntris", [20_000, 1_000_000])
def test_wide8_same_closest_t_as_reference(ctx_ref, ctx8, ntris):
    sc = synth.make_sized(23, ntris, env_size=(16, 8))
    bvh = Bvh.build(sc.vertices, sc.indices, 20)
    ds = DeviceScene(ctx_ref, sc.vertices, sc.indices, sc.materials, bvh)
    ds8 = DeviceScene(ctx8, sc.vertices, sc.indices, sc.materials, bvh)
    info = ds8.wide_bvh()
    assert info["width"] == 8 and info["nodes"] > 0 and 0 < info["levels"] <= 16, info
    rays = helpers.random_rays(sc.vertices, 200_000, seed=24)
    o = oracle_lib.Oracle()
    p = oracle_lib.make_params(sc.camera.matrix_world, sc.camera.fov, sc.camera.near, 640, 360)
    xy, r2 = helpers.camera_rays_ref(None, None, 640, 360, 100_000, seed=22)
    cam = o.camera_rays(p, xy, r2)
    crays = np.zeros((cam.shape[0], 8), np.float32)
    crays[:, :6], crays[:, 6] = cam, 1e5
    rays = np.concatenate([rays, crays])
    rtri, rt, ruv = trace_gpu(ctx_ref, ds, rays)
    tri, t, uv = trace_gpu(ctx8, ds8, rays)
    assert (rtri >= 0).sum() > 500
    check_same_t(tri, t, rtri, rt)
    same = tri == rtri
    np.testing.assert_array_equal(uv[same].view(np.uint32), ruv[same].view(np.uint32))
    np.testing.assert_array_equal(trace_gpu(ctx8, ds8, rays, True), trace_gpu(ctx_ref, ds, rays, True))
    ds.close()
    ds8.close()


def test_wide8_golden_with_documented_ties(ctx8):
    g = helpers.load_golden()
    bvh = Bvh(g["bvh_nodes"], g["bvh_indices"], 0, g["indices"].size // 3)
    ds = DeviceScene(ctx8, g["vertices"], g["indices"], g["materials"], bvh)
    assert ds.wide_bvh()["width"] == 8
    rays = g["rays"]
    tri, t, _ = trace_gpu(ctx8, ds, rays)
    ref_t, ref_tri = g["hit_t"], g["hit_tri"]
    np.testing.assert_array_equal(tri >= 0, ref_tri >= 0)
    differ = (tri >= 0) & (t.view(np.uint32) != ref_t.view(np.uint32))
    print(f"golden: {differ.sum()} of {(tri >= 0).sum()} hits at a different t (coplanar ties)")
    assert differ.mean() < 0.005
    if differ.any():
        rel = np.abs(t[differ].astype(np.float64) - ref_t[differ]) / np.abs(ref_t[differ].astype(np.float64))
        assert rel.max() <= TIE_REL, rel.max()
        o = oracle_lib.Oracle()
        o.set_scene(g["vertices"], g["indices"], g["materials"], g["bvh_nodes"], g["bvh_indices"])
        btri, bt, _, _ = o.trace(rays[differ], mode=1)  # brute force over every triangle
        np.testing.assert_array_equal(t[differ].view(np.uint32), bt.view(np.uint32))
    np.testing.assert_array_equal(trace_gpu(ctx8, ds, rays, True), g["occluded"])
    ds.close()


def test_wide8_degenerate_rays_take_the_binary_traversal(ctx_ref, ctx8):
    g = helpers.load_golden()
    bvh = Bvh(g["bvh_nodes"], g["bvh_indices"], 0, g["indices"].size // 3)
    ds = DeviceScene(ctx_ref, g["vertices"], g["indices"], g["materials"], bvh)
    ds8 = DeviceScene(ctx8, g["vertices"], g["indices"], g["materials"], bvh)
    rays = np.zeros((8, 8), np.float32)
    rays[:, 6] = 1e5
    rays[:, 0:3] = [0.4, 0.5, 0.45]
    rays[0, 3:6] = [0, 0, 0]           # zero direction: NaN slabs
    rays[1, 3:6] = [0, -1, 0]          # axis-aligned: infinite 1/d components
    rays[2, 3:6] = [1, 0, 0]
    rays[3, 3:6] = [0, 0, -1]
    rays[4, 3:6] = [0, -1, 0]; rays[4, 6] = 0.0   # tfar 0
    rays[5, 0:3] = [np.nan, 0, 0]; rays[5, 3:6] = [0, 1, 0]
    rays[6, 0:3] = [1e30, 1e30, 1e30]; rays[6, 3:6] = [-0.5, -0.5, -0.70710677]
    rays[7, 3:6] = [0.3, -0.8, 0.2]
    tri, t, _ = trace_gpu(ctx8, ds8, rays)
    rtri, rt, _ = trace_gpu(ctx_ref, ds, rays)
    # hit/miss and t bit for bit (the last ray meets two coplanar faces at exactly the same t)
    np.testing.assert_array_equal(tri >= 0, rtri >= 0)
    np.testing.assert_array_equal(t.view(np.uint32), rt.view(np.uint32))
    np.testing.assert_array_equal(trace_gpu(ctx8, ds8, rays, True), trace_gpu(ctx_ref, ds, rays, True))
    ds.close()
    ds8.close()


def test_wide8_leaf_root_keeps_the_4_wide_tree(ctx8):
    # one triangle: the binary root is a leaf, which has no box to quantise
    v = np.zeros((3, 20), np.float32)
    v[:, 0:3] = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    v[:, 6] = 1.0
    ds = DeviceScene(ctx8, v, np.array([0, 1, 2], np.uint32), synth.default_material()[None])
    assert ds.wide_bvh()["width"] == 4
    rays = np.zeros((2, 8), np.float32)
    rays[:, 0:3] = [0.2, 0.2, 1.0]
    rays[:, 3:6] = [0, 0, -1]
    rays[:, 6] = 1e5
    tri, t, _ = trace_gpu(ctx8, ds, rays)
    assert (tri == 0).all() and np.allclose(t, 1.0)
    ds.close()


@pytest.mark.parametrize("builder", ["host", "device", "device_lbvh"])
def test_wide8_after_refit(builder):
    sc = synth.make_sized(7, 30000, env_size=(16, 8))
    ctx = wide8_context(builder)
    ds = DeviceScene(ctx, sc.vertices, sc.indices, sc.materials)
    assert ds.wide_bvh()["width"] == 8
    moved = _deform(sc.vertices)
    ds.update_vertices(moved)
    assert ds.wide_bvh()["width"] == 8
    rays = helpers.random_rays(moved, 20000, seed=8)
    tri, t, _ = trace_gpu(ctx, ds, rays)
    set_traversal(ctx, _lib.TRAVERSAL_REFERENCE)
    rtri, rt, _ = trace_gpu(ctx, ds, rays)
    set_traversal(ctx, _lib.TRAVERSAL_WIDE)
    check_same_t(tri, t, rtri, rt)
    np.testing.assert_array_equal(trace_gpu(ctx, ds, rays, True) != 0, rtri >= 0)
    ds.close()
    ctx.close()


def test_wide8_image_matches_oracle_per_pixel():
    sc = synth.make_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    W, H, F = 128, 128, 8
    v = PathtracingViewport(width=W, height=H, settings={"maxBounces": 8, "envSampling": "cdf", "traversal": "wide"})
    v.ctx.set_wide_bvh(8)
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(PathtracingCamera(sc.camera.matrix_world, sc.camera.fov, sc.camera.near))
    assert v._scene.wide_bvh()["width"] == 8
    v.start(F)
    img = v.readAccumulation()
    d = v.diagnostics
    v.dispose()
    assert d["sample_count"] == F and d["traversal_aborted"] == 0
    o = oracle_lib.Oracle()
    o.set_scene(sc.vertices, sc.indices, sc.materials, sc.bvh.nodes, sc.bvh.indices)
    o.set_ibl(sc.env)
    p = oracle_lib.make_params(sc.camera.matrix_world, sc.camera.fov, sc.camera.near, W, H, max_bounces=8)
    ref = o.render_image(p, F)
    close = helpers.close_mask(img[..., :3], ref[..., :3], 1e-3, 1e-4).all(-1)
    print("pixels equal path for path:", close.mean())
    assert close.mean() >= 0.999
