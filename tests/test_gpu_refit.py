"""BVH refit on the device (dspbr_scene_update_vertices): after the vertices
move, the refitted binary tree gives the reference traversal's closest hits
bit for bit (against the oracle over the read-back tree and the new
vertices), the 4-wide tree the same closest t, and both agree with a scene
built from scratch over the new vertices."""
import numpy as np
import pytest

from dspbr import _lib, synth
from dspbr.viewport import Bvh, Context, DeviceScene, PathtracingViewport
from oracle import oracle_lib
from tests import helpers
from tests.test_gpu_parity import set_traversal, trace_gpu

pytestmark = pytest.mark.gpu


def _deform(v, k=0.6, seed=0):
    """Moves every position by a smooth field (normals kept)."""
    rng = np.random.default_rng(seed)
    out = v.copy()
    p = v[:, :3].astype(np.float64)
    span = p.max(0) - p.min(0)
    ph = rng.uniform(0, 2 * np.pi, 3)
    for a in range(3):
        out[:, a] = (p[:, a] + k * 0.05 * span[a] * np.sin(3.0 * p[:, (a + 1) % 3] / max(span[(a + 1) % 3], 1e-6)
                                                           * 2 * np.pi + ph[a])).astype(np.float32)
    return out


@pytest.mark.parametrize("builder", ["host", "device", "device_lbvh"])
def test_refit_hits_match_reference_traversal_and_a_fresh_build(builder):
    sc = synth.make_sized(7, 30000, env_size=(16, 8))
    ctx = Context(0)
    ctx.set_bvh_builder(builder)
    ds = DeviceScene(ctx, sc.vertices, sc.indices, sc.materials)
    moved = _deform(sc.vertices)
    ds.update_vertices(moved)
    bvh = ds.bvh()
    rays = helpers.random_rays(moved, 20000, seed=8)
    # reference traversal over the refitted tree = the oracle over the same tree and vertices
    set_traversal(ctx, _lib.TRAVERSAL_REFERENCE)
    rtri, rt, _ = trace_gpu(ctx, ds, rays)
    o = oracle_lib.Oracle()
    o.set_scene(moved, sc.indices, sc.materials, bvh.nodes, bvh.indices)
    otri, ot, _, st = o.trace(rays, mode=0)
    assert st["aborted"] == 0
    np.testing.assert_array_equal(rtri, otri)
    np.testing.assert_array_equal(rt.view(np.uint32), ot.view(np.uint32))
    # brute force over the new vertices: the refitted tree misses nothing
    btri, bt, _, _ = o.trace(rays, mode=1)
    np.testing.assert_array_equal(rtri >= 0, btri >= 0)
    np.testing.assert_array_equal(rt[rtri >= 0].view(np.uint32), bt[btri >= 0].view(np.uint32))
    # the 4-wide tree: the same closest t
    set_traversal(ctx, _lib.TRAVERSAL_WIDE)
    wtri, wt, _ = trace_gpu(ctx, ds, rays)
    np.testing.assert_array_equal(wtri >= 0, rtri >= 0)
    np.testing.assert_array_equal(wt.view(np.uint32), rt.view(np.uint32))
    assert (wtri != rtri).mean() < 1e-3  # exact t-ties only
    # a scene built from scratch over the new vertices finds the same hits
    fresh = DeviceScene(ctx, moved, sc.indices, sc.materials)
    ftri, ft, _ = trace_gpu(ctx, fresh, rays)
    np.testing.assert_array_equal(ft.view(np.uint32), wt.view(np.uint32))
    # occlusion from the refitted trees
    occ = trace_gpu(ctx, ds, rays, any_hit=True)
    np.testing.assert_array_equal(occ != 0, wtri >= 0)
    for d in (ds, fresh):
        d.close()
    ctx.close()


def test_partial_update_and_render_after_refit():
    sc = synth.make_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    moved = sc.vertices.copy()
    first, count = 100, 200
    moved[first:first + count, 1] += 0.25  # lift a part of the mesh
    # render after a partial update = render of a scene created over the moved vertices with the
    # refitted tree (reference binary traversal: the same tree, so the same paths)
    v = PathtracingViewport(width=48, height=40, settings={"maxBounces": 6, "traversal": "reference"})
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(helpers.camera_of(sc))
    v.start(2)
    v._scene.update_vertices(moved[first:first + count], first)
    d = v.diagnostics
    assert d["sample_count"] == 0  # the update reset the accumulation
    v.start(3)
    img = v.readAccumulation()
    bvh = v._scene.bvh()
    v.dispose()
    ref_scene = synth.Scene("moved", moved, sc.indices, sc.materials, sc.camera, env=sc.env)
    ref_scene.bvh = bvh  # the refitted tree, uploaded as a prebuilt BVH
    w = PathtracingViewport(width=48, height=40, settings={"maxBounces": 6, "traversal": "reference"})
    w.setScene(ref_scene)
    w.setIBL(sc.env)
    w.setCamera(helpers.camera_of(sc))
    w.start(3)
    ref = w.readAccumulation()
    w.dispose()
    np.testing.assert_allclose(img, ref, rtol=1e-6, atol=1e-7)
    with pytest.raises(_lib.DspbrError):
        c = Context(0)
        ds = DeviceScene(c, sc.vertices, sc.indices, sc.materials, sc.bvh)
        try:
            ds.update_vertices(moved[:10], sc.vertices.shape[0] - 5)  # past the end
        finally:
            ds.close()
            c.close()
