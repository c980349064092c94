"""BVH built on the device (DSPBR_BVH_BUILD_DEVICE: binned SAH;
DSPBR_BVH_BUILD_DEVICE_LBVH: linear BVH): a valid tree in the reference
layout, the same closest hits as the host-built tree, and the same images."""
import time

import numpy as np
import pytest

from dspbr import synth
from dspbr.viewport import Bvh, Context, DeviceScene, PathtracingViewport
from oracle import oracle_lib
from tests import helpers

pytestmark = pytest.mark.gpu


def _leaves(bvh: Bvh):
    """Slot ranges of the leaves reachable from the root (reference layout)."""
    nodes = bvh.nodes.reshape(-1, 16)
    out, stack = [], [0]
    while stack:
        n = stack.pop()
        cnt, first = int(nodes[n, 11]), int(nodes[n, 15])
        if cnt > 0:
            out.append((first, cnt))
        else:
            stack += [int(nodes[n, 3]), int(nodes[n, 7])]
    return out


# the largest leaf each builder makes (SAH: the host builder's leaf cap)
MAX_LEAF = {"device": 8, "device_lbvh": 4}


@pytest.mark.parametrize("builder", ["device", "device_lbvh"])
@pytest.mark.parametrize("ntris", [1, 7, 3000, 200_000])
def test_device_bvh_is_a_valid_reference_layout_tree(ntris, builder):
    sc = synth.make_sized(41, max(ntris, 20), env_size=(16, 8)) if ntris > 7 else synth.make_small(0)
    if ntris <= 7:  # a tiny mesh: the first `ntris` triangles of the small scene
        sc.indices = np.ascontiguousarray(sc.indices[: 3 * ntris])
    ctx = Context(0)
    ctx.set_bvh_builder(builder)
    ds = DeviceScene(ctx, sc.vertices, sc.indices, sc.materials)
    bvh = ds.bvh()
    n = sc.indices.size // 3
    # every triangle in exactly one reachable leaf, leaves of at most the builder's size
    seen = np.zeros(n, np.int32)
    for first, cnt in _leaves(bvh):
        assert 1 <= cnt <= MAX_LEAF[builder]
        seen[bvh.indices[first:first + cnt]] += 1
    assert (seen == 1).all()
    # closest hits of the reference traversal over it = brute force (ties aside)
    o = oracle_lib.Oracle()
    o.set_scene(sc.vertices, sc.indices, sc.materials, bvh.nodes, bvh.indices)
    rays = helpers.random_rays(sc.vertices, 3000, seed=42)
    tri, t, _, st = o.trace(rays, mode=0)
    btri, bt, _, _ = o.trace(rays, mode=1)
    assert st["aborted"] == 0
    np.testing.assert_array_equal(tri >= 0, btri >= 0)
    np.testing.assert_array_equal(t[tri >= 0].view(np.uint32), bt[btri >= 0].view(np.uint32))
    ds.close()
    ctx.close()


@pytest.mark.parametrize("builder", ["device", "device_lbvh"])
def test_device_bvh_same_hits_and_image_as_host_bvh(builder):
    sc = synth.make_sized(43, 400_000, env_size=(64, 32))
    hc, dc = Context(0), Context(0)
    dc.set_bvh_builder(builder)
    t0 = time.perf_counter()
    hs = DeviceScene(hc, sc.vertices, sc.indices, sc.materials)
    t1 = time.perf_counter()
    ds = DeviceScene(dc, sc.vertices, sc.indices, sc.materials)
    t2 = time.perf_counter()
    print(f"scene creation: host SAH {t1 - t0:.3f} s, {builder} {t2 - t1:.3f} s")
    from tests.test_gpu_parity import trace_gpu
    rays = helpers.random_rays(sc.vertices, 100_000, seed=44)
    htri, ht, _ = trace_gpu(hc, hs, rays)
    dtri, dt, _ = trace_gpu(dc, ds, rays)
    np.testing.assert_array_equal(htri >= 0, dtri >= 0)
    np.testing.assert_array_equal(ht.view(np.uint32), dt.view(np.uint32))
    assert (htri != dtri).mean() < 1e-3
    np.testing.assert_array_equal(trace_gpu(hc, hs, rays, True), trace_gpu(dc, ds, rays, True))
    for o in (hs, ds):
        o.close()
    hc.close()
    dc.close()
    imgs = []
    for b in ("host", builder):
        v = PathtracingViewport(width=96, height=64, settings={"maxBounces": 6, "bvhBuilder": b})
        v.setScene(sc)
        v.setIBL(sc.env)
        v.setCamera(helpers.camera_of(sc))
        v.start(2)
        imgs.append(v.readAccumulation())
        v.dispose()
    close = helpers.close_mask(imgs[0][..., :3], imgs[1][..., :3], 1e-4, 1e-5).all(-1)
    assert close.mean() > 0.99


def _canonical(bvh: Bvh):
    """The tree from the root as nested tuples: inner nodes by their two
    child boxes (float bits), leaves by their sorted triangle ids, so that
    trees numbered in different orders compare equal."""
    nodes = bvh.nodes.reshape(-1, 16)
    bits = nodes.view(np.uint32)

    def walk(n):
        cnt, first = int(nodes[n, 11]), int(nodes[n, 15])
        if cnt > 0:
            return ("leaf", tuple(sorted(int(t) for t in bvh.indices[first:first + cnt])))
        boxes = tuple(int(x) for k in (0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14) for x in [bits[n, k]])
        return ("inner", boxes, walk(int(nodes[n, 3])), walk(int(nodes[n, 7])))

    import sys
    limit = sys.getrecursionlimit()
    sys.setrecursionlimit(max(limit, 10_000))
    try:
        return walk(0)
    finally:
        sys.setrecursionlimit(limit)


@pytest.mark.parametrize("ntris", [3000, 60_000])
def test_device_sah_builds_the_host_tree(ntris):
    """The device binned SAH applies the host builder's rules: the same tree
    (structure, child boxes bit for bit, leaf triangle sets)."""
    sc = synth.make_sized(47, ntris, env_size=(16, 8))
    host = Bvh.build(sc.vertices, sc.indices)
    ctx = Context(0)
    ctx.set_bvh_builder("device")
    ds = DeviceScene(ctx, sc.vertices, sc.indices, sc.materials)
    dev = ds.bvh()
    assert dev.nodes.size == host.nodes.size
    assert _canonical(dev) == _canonical(host)
    ds.close()
    ctx.close()


def test_builder_selection_checks_its_argument():
    """dspbr_set_bvh_builder takes the three builder codes only; the Python
    mirror takes their names."""
    from dspbr import _lib
    ctx = Context(0)
    for code in (_lib.BVH_BUILD_HOST, _lib.BVH_BUILD_DEVICE, _lib.BVH_BUILD_DEVICE_LBVH):
        assert ctx.lib.dspbr_set_bvh_builder(ctx.h, code) == 0
    assert ctx.lib.dspbr_set_bvh_builder(ctx.h, 3) != 0
    assert ctx.lib.dspbr_set_bvh_builder(ctx.h, -1) != 0
    with pytest.raises(ValueError):
        ctx.set_bvh_builder("gpu")
    for name in ("host", "device", "device_lbvh"):
        ctx.set_bvh_builder(name)
    ctx.close()
