"""Render server (continuous batching): each request's image is the one it
renders alone and the one the single-viewport API renders; cancellation,
HBM-budget admission, autotuning and a mixed stream of requests."""
import numpy as np
import pytest

from dspbr import _lib, synth
from dspbr.server import Server
from dspbr.viewport import Bvh, Context, DeviceIbl, DeviceScene, PathtracingCamera, PathtracingViewport, look_at_matrix

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-6, atol=1e-7)  # FP64 pixel sums in a different order


@pytest.fixture(scope="module")
def world():
    ctx = Context(0)
    small = synth.make_small(0)
    small.bvh = Bvh.build(small.vertices, small.indices, 20)
    sized = synth.make_sized(3, 20000, env_size=(256, 128))
    sized.bvh = Bvh.build(sized.vertices, sized.indices, 20)
    scenes = [DeviceScene(ctx, s.vertices, s.indices, s.materials, s.bvh) for s in (small, sized)]
    ibls = [DeviceIbl(ctx, small.env), DeviceIbl(ctx, sized.env)]
    yield ctx, (small, sized), scenes, ibls
    for o in scenes + ibls:
        o.close()
    ctx.close()


def _cam(sc, k=0):
    if k == 0:
        return PathtracingCamera(sc.camera.matrix_world, sc.camera.fov, sc.camera.near)
    m = look_at_matrix((0.3 * k, 1.0, 3.0 + 0.2 * k), (0, 0.8, 0))
    return PathtracingCamera(m, 40.0 + 5 * k, 0.05)


def _requests(world):
    ctx, hosts, scenes, ibls = world
    return [
        dict(si=0, cam=0, w=64, h=48, spp=4, settings={"maxBounces": 6}),
        dict(si=1, cam=0, w=96, h=64, spp=3, settings={"maxBounces": 8, "envSampling": "cdf"}),
        dict(si=0, cam=1, w=33, h=17, spp=5, settings={"maxBounces": 4, "rng": "pcg", "seed": 9}),
        dict(si=1, cam=2, w=40, h=40, spp=2, settings={"maxBounces": 5, "materialProfile": "webgl-lean"}),
        dict(si=0, cam=3, w=7, h=3, spp=1, settings={"maxBounces": 3, "showBackground": False,
                                                      "backgroundColor": [0.2, 0.3, 0.4, 1.0]}),
    ]


def _submit(srv, world, r, out=None):
    ctx, hosts, scenes, ibls = world
    return srv.submit(scenes[r["si"]], ibls[r["si"]], _cam(hosts[r["si"]], r["cam"]), r["w"], r["h"], r["spp"],
                      r["settings"], out=out)


def test_request_alone_equals_mix_equals_viewport(world):
    ctx, hosts, scenes, ibls = world
    reqs = _requests(world)
    alone = []
    for r in reqs:
        srv = Server(ctx, path_pool=1 << 16)
        img, info = srv.wait(_submit(srv, world, r))
        assert info["state"] == "done"
        alone.append(img.copy())
        srv.close()
    # all at once, a pool smaller than the work (slots shared and refilled)
    srv = Server(ctx, path_pool=5000)
    pinned = ctx.host_array((reqs[1]["h"], reqs[1]["w"], 4))
    ids = [_submit(srv, world, r, out=pinned if i == 1 else None) for i, r in enumerate(reqs)]
    mix = []
    for rid in ids:
        img, info = srv.wait(rid, timeout_ms=120000)
        assert info["state"] == "done"
        mix.append(img.copy())
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for a, m in zip(alone, mix):
        np.testing.assert_allclose(m, a, **TOL)
        assert np.isfinite(a).all() and a[..., :3].max() > 0
    # the single-viewport API renders the same image
    r = reqs[0]
    v = PathtracingViewport(width=r["w"], height=r["h"], settings=r["settings"])
    v.setScene(hosts[r["si"]])
    v.setIBL(hosts[r["si"]].env)
    v.setCamera(_cam(hosts[r["si"]], r["cam"]))
    v.start(r["spp"])
    ref = v.readAccumulation()
    v.dispose()
    np.testing.assert_allclose(alone[0], ref, **TOL)


def test_cancel_and_queue_order(world):
    ctx, hosts, scenes, ibls = world
    srv = Server(ctx, path_pool=1 << 16)
    big = srv.submit(scenes[1], ibls[1], _cam(hosts[1]), 512, 512, 256, {"maxBounces": 8})
    small = srv.submit(scenes[0], ibls[0], _cam(hosts[0]), 16, 16, 2, {"maxBounces": 4})
    srv.cancel(big)
    _, ib = srv.wait(big, timeout_ms=120000)
    img, isml = srv.wait(small, timeout_ms=120000)
    assert ib["state"] == "cancelled"
    assert isml["state"] == "done" and np.isfinite(img).all()
    with pytest.raises(_lib.DspbrError):
        srv.release(12345)
    srv.release(big)
    with pytest.raises(_lib.DspbrError):
        srv.poll(big)
    srv.close()


def test_hbm_budget_admission(world):
    ctx, hosts, scenes, ibls = world
    srv = Server(ctx, path_pool=1 << 12, hbm_budget_bytes=1 << 20)
    with pytest.raises(_lib.DspbrError) as e:
        srv.submit(scenes[0], ibls[0], _cam(hosts[0]), 1024, 1024, 1)
    assert e.value.code == -5
    srv.close()
    # a budget that holds one 128x128 request at a time: the second waits for the first
    pool_and_scene = Server(ctx, path_pool=1 << 12)
    base = pool_and_scene.stats()["bytes_in_use"] + scenes[0].device_bytes()
    pool_and_scene.close()
    one = 128 * 128 * 48
    srv = Server(ctx, path_pool=1 << 12, hbm_budget_bytes=base + one + one // 2)
    a = srv.submit(scenes[0], ibls[0], _cam(hosts[0]), 128, 128, 8, {"maxBounces": 6})
    b = srv.submit(scenes[0], ibls[0], _cam(hosts[0], 1), 128, 128, 8, {"maxBounces": 6})
    _, ia = srv.wait(a, timeout_ms=120000)
    _, ib = srv.wait(b, timeout_ms=120000)
    assert ia["state"] == ib["state"] == "done"
    assert ib["admit_ms"] >= ia["done_ms"] - 50.0  # admitted once a's buffers were released
    st = srv.stats()
    assert st["bytes_peak"] <= base + one + one // 2
    srv.close()


def test_autotune_then_serve(world, tmp_path):
    ctx, hosts, scenes, ibls = world
    srv = Server(ctx)
    samples = [srv.request(scenes[i], ibls[i], _cam(hosts[i]), 256, 256, 4)[0] for i in (0, 1)]
    cache = str(tmp_path / "autotune.json")
    st = srv.autotune(samples, seconds=8.0, cache=cache)
    assert st["autotune_source"] == "tuned"
    assert st["path_pool"] in (1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24)
    assert st["trace_threads"] == 128 and st["shade_threads"] == 128
    sms = 148
    for k in ("trace_blocks", "connect_blocks", "shade_blocks"):
        assert st[k] % sms == 0 and sms <= st[k] <= 8 * sms, (k, st[k])
    chosen = srv.launch()
    r = _requests(world)[0]
    img, info = srv.wait(_submit(srv, world, r))
    srv.close()
    # a second server on the same GPU takes the cached choice without tuning
    again = Server(ctx)
    st2 = again.autotune(samples, seconds=8.0, cache=cache)
    assert st2["autotune_source"] == "cache" and again.launch() == chosen
    with pytest.raises(_lib.DspbrError):
        again.set_launch(dict(chosen, extend_blocks=chosen["extend_blocks"] + 1))  # not a multiple of the SMs
    again.close()
    ref_srv = Server(ctx, path_pool=1 << 16)
    ref, _ = ref_srv.wait(_submit(ref_srv, world, r))
    ref_srv.close()
    assert info["state"] == "done"
    np.testing.assert_allclose(img, ref, **TOL)


def test_mixed_stream_latency_stats(world):
    ctx, hosts, scenes, ibls = world
    rng = np.random.default_rng(5)
    srv = Server(ctx, path_pool=1 << 18)
    ids, specs = [], []
    for k in range(40):
        si = int(rng.integers(0, 2))
        w, h = int(rng.integers(8, 160)), int(rng.integers(8, 120))
        spp = int(rng.integers(1, 9))
        specs.append((si, k % 4, w, h, spp))
        ids.append(srv.submit(scenes[si], ibls[si], _cam(hosts[si], k % 4), w, h, spp, {"maxBounces": 6}))
    imgs = [srv.wait(i, timeout_ms=300000) for i in ids]
    st = srv.stats()
    srv.close()
    assert all(info["state"] == "done" for _, info in imgs)
    assert st["completed"] == 40 and st["p99_ms"] >= st["p50_ms"] > 0
    # spot-check three of them alone
    for k in (0, 17, 39):
        si, cam, w, h, spp = specs[k]
        s1 = Server(ctx, path_pool=1 << 14)
        ref, _ = s1.wait(s1.submit(scenes[si], ibls[si], _cam(hosts[si], cam), w, h, spp, {"maxBounces": 6}))
        s1.close()
        np.testing.assert_allclose(imgs[k][0], ref, **TOL)
