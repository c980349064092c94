"""The engine's render loop on the GPU: a render call runs as one graph (a
device-side while loop over pairs of iterations, then the tail drain), with
the same image as the host-driven loop of the profiling mode, and the
per-iteration timeline it records."""
import ctypes as C

import numpy as np
import pytest

from dspbr import synth
from dspbr.viewport import Bvh, PathtracingViewport
from tests import helpers

pytestmark = pytest.mark.gpu


def _viewport(settings):
    sc = synth.make_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    v = PathtracingViewport(width=96, height=64, settings=settings)
    v.setScene(sc)
    v.setIBL(sc.env)
    v.setCamera(helpers.camera_of(sc))
    return v


@pytest.mark.parametrize("pool", [0, 997, 20000])
def test_device_loop_equals_host_loop(pool):
    imgs = []
    for profiling in (0, 1):
        v = _viewport({"maxBounces": 8})
        if pool:
            v.ctx.check(v.ctx.lib.dspbr_set_wave_paths(v.ctx.h, pool))
        v.ctx.check(v.ctx.lib.dspbr_set_profiling(v.ctx.h, profiling))
        v.start(3)
        v.start(5)  # a second call continues the accumulation up to 5 samples
        imgs.append(v.readAccumulation())
        d = v.diagnostics
        v.dispose()
        assert d["sample_count"] == 5 and d["traversal_aborted"] == 0
    np.testing.assert_allclose(imgs[0], imgs[1], rtol=1e-6, atol=1e-7)


def test_timeline_of_a_render_call():
    v = _viewport({"maxBounces": 8})
    v.start(1)
    first = v.timeline(1)
    v.start(5)
    tl = v.timeline(1024)
    v.dispose()
    tl = tl[tl[:, 0] > first[-1, 0]]
    assert len(tl) >= 2
    assert (np.diff(tl[:, 0]) == 1).all() and (np.diff(tl[:, 1]) >= 0).all()
    assert tl[-1, 2] == 0  # the tail left no path


def test_resize_keeps_larger_buffers_and_images_match_a_fresh_viewport():
    """A viewport that grows, then shrinks, keeps its image buffers (they only
    grow) and renders what a viewport created at each size renders."""
    sizes = [(96, 64), (160, 100), (48, 32)]
    v = _viewport({"maxBounces": 8})
    got, disp = [], []
    for w, h in sizes:
        v.resize(w, h)
        v.start(3)
        got.append(v.readAccumulation().copy())
        disp.append(v.readDisplay().copy())
    v.dispose()
    for (w, h), img, d in zip(sizes, got, disp):
        f = _viewport({"maxBounces": 8})
        f.resize(w, h)
        f.start(3)
        assert img.shape[:2] == (h, w)
        # samples of one pixel are summed by atomics in completion order
        np.testing.assert_allclose(img, f.readAccumulation(), rtol=1e-6, atol=1e-7)
        assert np.abs(d.astype(np.int16) - f.readDisplay().astype(np.int16)).max() <= 1
        f.dispose()


def test_async_readback_overlapping_the_next_render():
    """read_accum_async: the mean of the frames rendered before the call,
    bit-equal to read_accum, although the next render runs during the copy;
    a read that follows is ordered after the pending copy; pageable memory is
    refused."""
    v = _viewport({"maxBounces": 8})
    v.start(3)
    ref3 = v.readAccumulation()
    bufs = [v.allocReadbackBuffer(), v.allocReadbackBuffer()]
    v.readAccumulationAsync(bufs[0])
    v.start(5)  # two more frames while the copy runs
    ref5 = v.readAccumulation()  # writes the mean buffer after the pending copy
    v.readWait()
    np.testing.assert_array_equal(bufs[0], ref3)
    v.readAccumulationAsync(bufs[1])
    v.readAccumulationAsync(bufs[0])  # a second pending copy of the same frames
    v.readWait()
    np.testing.assert_array_equal(bufs[1], ref5)
    np.testing.assert_array_equal(bufs[0], ref5)
    with pytest.raises(RuntimeError):
        v.readAccumulationAsync(np.empty_like(ref5))
    v.readAccumulationAsync(bufs[1])
    v.resize(48, 32)  # waits for the copy before the buffers can change
    np.testing.assert_array_equal(bufs[1], ref5)
    v.dispose()


def _one_frame(threshold):
    v = _viewport({"maxBounces": 8})
    v.ctx.check(v.ctx.lib.dspbr_set_drain_threshold(v.ctx.h, int(threshold)))
    v.start(1)
    tl = v.timeline(1024)
    img = v.readAccumulation()
    v.dispose()
    return img, tl


def test_tail_after_an_iteration_of_either_parity():
    """The render loop graph stops after whichever iteration first leaves
    fewer live paths than the drain threshold, and runs the tail of that
    iteration's parity; one sample per pixel, so the image is the same bits
    whichever iteration the tail starts after."""
    ref, tl = _one_frame(1)  # below 1 live path: no drain before the end
    live = [int(x) for x in tl[:, 2]]
    k = next(i for i in range(1, len(live) - 1) if live[i] > 0 and live[i + 1] > 0)
    counts = []
    for thr in (live[k] + 1, live[k + 1] + 1):  # the tail after iteration k, then k + 1
        img, t = _one_frame(thr)
        counts.append(len(t))
        np.testing.assert_array_equal(img, ref)
    assert counts[1] == counts[0] + 1  # consecutive iterations: both parities
