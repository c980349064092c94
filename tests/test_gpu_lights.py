"""The point light (lighting.glsl:2-22, misptdl.glsl:24-30) that the first scene
light sets (renderer.ts:424-430), on the GPU against the reference shaders'
golden image, through the viewport and through the server."""
import numpy as np
import pytest

from dspbr import synth
from dspbr.server import Server
from dspbr.viewport import Bvh, Context, DeviceIbl, DeviceScene, PathtracingViewport
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    return helpers.load_golden()


def _lit_scene(g):
    sc = synth.make_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    pos, emis = g["pl_light"]
    sc.lights = [{"position": tuple(pos), "type": 0, "emission": tuple(emis)}]
    return sc


@pytest.mark.parametrize("traversal", ["reference", "wide"])
def test_point_light_image_matches_golden_path_for_path(g, traversal):
    sc = _lit_scene(g)
    W, H, F = (int(x) for x in g["pl_image_whf"])
    v = PathtracingViewport(width=W, height=H, settings={"maxBounces": 8, "envSampling": "cdf",
                                                        "traversal": traversal})
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(helpers.camera_of(sc))
    v.start(F)
    img = v.readAccumulation()
    # the same viewport without the light renders the unlit golden image's scene
    sc.lights = []
    v.setScene(sc)
    v.start(F)
    unlit = v.readAccumulation()
    v.dispose()
    ref = g["pl_image"]
    close = helpers.close_mask(img[..., :3], ref[..., :3], 1e-3, 1e-4).all(-1)
    print("lit pixels equal to the reference path for path:", close.mean())
    assert close.mean() >= 0.999  # measured 1.0
    assert np.abs(img - ref).mean() < 0.01 * ref[..., :3].mean()
    assert unlit[..., :3].mean() < 0.95 * img[..., :3].mean()


def test_server_request_takes_the_scene_light(g):
    sc = _lit_scene(g)
    ctx = Context(0)
    ds = DeviceScene(ctx, sc.vertices, sc.indices, sc.materials, sc.bvh, lights=sc.lights)
    ibl = DeviceIbl(ctx, sc.env)
    W, H, F = (int(x) for x in g["pl_image_whf"])
    srv = Server(ctx, path_pool=1 << 14)
    img, info = srv.wait(srv.submit(ds, ibl, helpers.camera_of(sc), W, H, F,
                                    {"maxBounces": 8, "envSampling": "cdf"}))
    srv.close()
    v = PathtracingViewport(width=W, height=H, settings={"maxBounces": 8, "envSampling": "cdf"})
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(helpers.camera_of(sc))
    v.start(F)
    ref = v.readAccumulation()
    v.dispose()
    for o in (ds, ibl):
        o.close()
    ctx.close()
    assert info["state"] == "done"
    np.testing.assert_allclose(img, ref, rtol=1e-6, atol=1e-7)
