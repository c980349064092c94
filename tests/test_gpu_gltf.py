"""A glTF asset packed by dspbr.gltf (scene_loader.ts) and rendered on the GPU,
path for path against the reference shaders rendering the same packed scene."""
import numpy as np
import pytest

from dspbr import gltf, synth
from dspbr.viewport import Bvh, PathtracingCamera, PathtracingViewport
from tests import helpers
from dspbr.gltf_writer import sample_camera, sample_scene
from tests.test_gltf import packed_sha

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("traversal", ["reference", "wide"])
def test_gltf_scene_matches_golden_path_for_path(traversal):
    g = helpers.load_golden()
    sc = gltf.load_gltf(sample_scene().glb_bytes())
    assert packed_sha(sc) == bytes(g["gltf_vertices_sha"])  # the same packed buffers as the golden render
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    cam = sample_camera()
    W, H, F = (int(x) for x in g["gltf_image_whf"])
    v = PathtracingViewport(width=W, height=H, settings={"maxBounces": 8, "envSampling": "cdf",
                                                        "traversal": traversal})
    v.setScene(sc)
    v.setIBL(synth.make_small(0).env)
    v.setCamera(PathtracingCamera(cam.matrix_world, cam.fov, cam.near))
    v.start(F)
    img = v.readAccumulation()
    v.dispose()
    ref = g["gltf_image"]
    close = helpers.close_mask(img[..., :3], ref[..., :3], 1e-3, 1e-4).all(-1)
    print("glTF pixels equal to the reference path for path:", close.mean())
    assert close.mean() >= 0.999  # measured 1.0
    assert np.abs(img - ref).mean() < 0.01 * ref[..., :3].mean()
