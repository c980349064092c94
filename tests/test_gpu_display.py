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


def nearest_canvas(img, dw, dh):
    """display.frag's draw of a w x h buffer on a dw x dh canvas: NEAREST at
    uv = (x + 0.5) / dw, CLAMP_TO_EDGE (gl_utils.ts:22-33), in float32."""
    h, w = img.shape[:2]
    u = (np.arange(dw, dtype=np.float32) + np.float32(0.5)) / np.float32(dw)
    v = (np.arange(dh, dtype=np.float32) + np.float32(0.5)) / np.float32(dh)
    i = np.clip(np.floor(u * np.float32(w)).astype(np.int64), 0, w - 1)
    j = np.clip(np.floor(v * np.float32(h)).astype(np.int64), 0, h - 1)
    return img[j[:, None], i[None, :]]


def test_interaction_mode_renders_at_the_interaction_pixel_ratio(g):
    """setInteractionMode(true) renders at interactionPixelRatio of the canvas
    and restarts the accumulation; the displayed canvas is the render-size
    postprocess buffer drawn at the canvas size (display.frag)."""
    sc = synth.make_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    v = PathtracingViewport(width=67, height=45, settings={"maxBounces": 4, "toneMapping": "AcesFilm"})
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(helpers.camera_of(sc))
    v.start(2)
    full = v.readAccumulation()
    assert full.shape == (45, 67, 4)
    v.setInteractionMode(True)
    d = v.diagnostics
    assert d["sample_count"] == 0 and d["renderResolution"] == "34x23" and d["displayResolution"] == "67x45"
    v.start(3)
    low = v.readAccumulation()
    assert low.shape == (23, 34, 4) and v.diagnostics["rays_primary"] == 67 * 45 * 2 + 34 * 23 * 3
    shown = v.readDisplay(rgba8=False)
    shown8 = v.readDisplay()
    assert shown.shape == (45, 67, 4) and shown8.shape == (45, 67, 4)
    c = Context(0)
    ref, ref8 = display(c, low, 3, gamma=True)
    c.close()
    np.testing.assert_array_equal(shown, nearest_canvas(ref, 67, 45))
    np.testing.assert_array_equal(shown8, nearest_canvas(ref8, 67, 45))
    # the same camera at half resolution: the low image is the half-resolution render
    h = PathtracingViewport(width=34, height=23, settings={"maxBounces": 4})
    h.setScene(sc)
    h.setIBL(sc.env)
    h.setCamera(helpers.camera_of(sc))
    h.start(3)
    np.testing.assert_allclose(low, h.readAccumulation(), rtol=1e-6, atol=1e-7)
    h.dispose()
    # back to pixelRatio 1: full resolution, accumulation restarted
    v.setInteractionMode(False)
    assert v.diagnostics["sample_count"] == 0 and v.diagnostics["renderResolution"] == "67x45"
    v.start(2)
    np.testing.assert_allclose(v.readAccumulation(), full, rtol=1e-6, atol=1e-7)
    v.dispose()
