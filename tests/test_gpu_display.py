"""Display epilogue (tonemap.frag, fxaa.frag, 8-bit canvas) on the GPU against
golden vectors made by the reference's own shaders compiled for the host."""
import ctypes as C

import numpy as np
import pytest

from dspbr import _lib, synth
from dspbr.viewport import Bvh, Context, PathtracingViewport
from tests import helpers

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def g():
    return helpers.load_golden()


def display(ctx, img, mode, exposure=1.0, gamma=True, fxaa=False):
    img = np.ascontiguousarray(img, np.float32)
    h, w = img.shape[:2]
    d = _lib.Display()
    d.exposure, d.tonemapping, d.gamma, d.fxaa = exposure, mode, int(gamma), int(fxaa)
    out = np.zeros_like(img)
    out8 = np.zeros((h, w, 4), np.uint8)
    ctx.check(ctx.lib.dspbr_display_image(ctx.h, _lib.fptr(img), w, h, C.byref(d), _lib.fptr(out),
                                          out8.ctypes.data_as(C.POINTER(C.c_uint8))))
    return out, out8


def ulps(a, b):
    ia = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    ib = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


def canvas(x):
    return np.rint(np.clip(x, 0.0, 1.0) * 255.0).astype(np.int32)


@pytest.mark.parametrize("gamma", [0, 1])
def test_tonemap_modes_match_reference(ctx, g, gamma):
    hdr = g["display_hdr"]
    for k, mode in enumerate(g["display_modes"]):
        ref = g[f"display_tonemap_g{gamma}"][k]
        out, out8 = display(ctx, hdr, int(mode), exposure=1.7, gamma=bool(gamma))
        if gamma == 0 and mode != 2:
            # no pow(): every operation rounds as in the shader
            np.testing.assert_array_equal(out, ref, err_msg=f"mode {mode}")
        else:
            # pow() of the CUDA math library vs the host libm: a few ulps
            assert ulps(out, ref).max() <= 4, f"mode {mode}: {ulps(out, ref).max()} ulps"
        d8 = np.abs(out8.astype(np.int32) - canvas(ref))
        assert d8.max() <= 1 and (d8 == 0).mean() > 0.999, f"mode {mode}"


def test_fxaa_matches_reference(ctx, g):
    tm = g["display_fxaa_in"]
    # FXAA on the reference's tone-mapped image: exposure 1, no operator, no gamma
    out, out8 = display(ctx, tm, -1, gamma=False, fxaa=True)
    np.testing.assert_array_equal(out, g["display_fxaa"])
    assert (out != tm).any()  # the pass changed edge pixels
    np.testing.assert_array_equal(out8.astype(np.int32), canvas(g["display_fxaa"]))


def test_aces_fxaa_of_rendered_image(ctx, g):
    out, _ = display(ctx, g["image"], 3, gamma=True, fxaa=True)
    ref = g["display_image_aces_fxaa"]
    assert ulps(out, ref).max() <= 4


def test_viewport_read_display(g):
    sc = synth.make_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    v = PathtracingViewport(width=64, height=48, settings={"maxBounces": 6, "toneMapping": "AcesFilm",
                                                          "exposure": 1.3, "enableFxaa": True})
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(helpers.camera_of(sc))
    v.start(3)
    acc = v.readAccumulation()
    shown = v.readDisplay(rgba8=False)
    shown8 = v.readDisplay()
    v.setSettings({"toneMapping": "Filmic"})  # not in tonemappingModes: no operator (index -1)
    raw = v.readDisplay(rgba8=False)
    v.dispose()
    c = Context(0)
    ref, ref8 = display(c, acc, 3, exposure=1.3, gamma=True, fxaa=True)
    ref_raw, _ = display(c, acc, -1, exposure=1.3, gamma=True, fxaa=True)
    c.close()
    np.testing.assert_array_equal(shown, ref)
    np.testing.assert_array_equal(shown8, ref8)
    np.testing.assert_array_equal(raw, ref_raw)
    assert shown8.dtype == np.uint8 and shown8[..., 3].min() == 255
