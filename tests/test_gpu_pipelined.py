"""Pipelined frames (dspbr_set_pipelining, dspbr_set_pipeline_depth): the
render of one accumulation overlaps the tail of the previous one (or two) on
the device.  Every image must equal
the image of the same calls without pipelining (FP64 pixel sums in another
order: allclose 1e-6), whatever mix of camera changes, progressive renders,
asynchronous and synchronous reads, display reads and resizes comes."""
import ctypes as C

import numpy as np
import pytest

from dspbr import synth
from dspbr.viewport import Bvh, PathtracingCamera, PathtracingViewport, look_at_matrix

pytestmark = pytest.mark.gpu

TOL = dict(rtol=1e-6, atol=1e-7)


@pytest.fixture(scope="module")
def scene():
    sc = synth.make_small(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    return sc


def _viewport(sc, pipelined, w=96, h=64, pool=0):
    v = PathtracingViewport(width=w, height=h, settings={"maxBounces": 8, "pipelinedFrames": pipelined})
    if pool:
        v.ctx.check(v.ctx.lib.dspbr_set_wave_paths(v.ctx.h, pool))
    v.setScene(sc)
    v.setIBL(sc.env)
    return v


def _cam(k):
    return PathtracingCamera(look_at_matrix((0.25 * k - 0.5, 1.0, 3.4 - 0.1 * k), (0, 0.9, 0)), 45.0, 0.1)


@pytest.mark.parametrize("pool", [0, 4000])
@pytest.mark.parametrize("mode", [True, 3, 16])
def test_camera_per_frame_with_async_reads(scene, pool, mode):
    """The interactive loop: per frame setCamera, start(1), then the previous
    frame's readWait and this frame's readAccumulationAsync."""
    out = {}
    for pipelined in (False, mode):
        v = _viewport(scene, pipelined, pool=pool)
        bufs = [v.allocReadbackBuffer() for _ in range(6)]
        for k in range(6):
            v.setCamera(_cam(k))
            v.start(1)
            assert v.diagnostics["sample_count"] == 1
            v.readWait()
            v.readAccumulationAsync(bufs[k])
        v.readWait()
        out[pipelined] = [b.copy() for b in bufs]
        d = v.diagnostics
        assert d["rays_primary"] == 6 * 96 * 64 and d["traversal_aborted"] == 0
        v.dispose()
    for a, b in zip(out[False], out[mode]):
        assert np.isfinite(b).all() and b[..., 3].min() == 1.0
        np.testing.assert_allclose(b, a, **TOL)
    # the frames differ (different cameras): the reads did not repeat one image
    assert not np.allclose(out[mode][0], out[mode][1])


def test_progressive_and_mixed_calls(scene):
    """Progressive renders that continue an accumulation in flight, a read of
    an accumulation in flight followed by more frames of it, a synchronous
    read, a display read, a resize and a reset with nothing rendered."""
    res = {}
    for pipelined in (False, True, 3, 16):
        v = _viewport(scene, pipelined)
        got = []
        v.setCamera(_cam(0))
        v.start(1)
        v.start(2)  # the same accumulation: 2 samples
        buf = v.allocReadbackBuffer()
        v.readAccumulationAsync(buf)
        v.start(4)  # two more samples after the read was requested
        v.readWait()
        got.append(buf.copy())  # the 2-sample mean
        got.append(v.readAccumulation())  # 4 samples
        v.setCamera(_cam(1))
        v.start(1)
        v.setCamera(_cam(2))  # a new accumulation while the last one is in flight ...
        v.resetAccumulation()  # ... and another reset with nothing rendered
        v.start(2)
        got.append(v.readDisplay(rgba8=False))
        v.resize(80, 48)
        v.setCamera(_cam(3))
        v.start(1)
        got.append(v.readAccumulation())
        assert v.diagnostics["sample_count"] == 1
        res[pipelined] = got
        v.dispose()
    for mode in (True, 3, 16):
        for a, b in zip(res[False], res[mode]):
            np.testing.assert_allclose(b, a, **TOL)


def _sample_count(v):
    n = C.c_ulonglong(0)
    v.ctx.check(v.ctx.lib.dspbr_get_sample_count(v.ctx.h, C.byref(n)))
    return n.value


def test_calls_while_a_render_loop_runs(scene):
    """A pipelined render call returns while its loop runs: the counter read
    without waiting, diagnostics (which wait for the loop), a settings change
    (a reset), a progressive continuation and a synchronous read right after
    it give what the same calls give without pipelining."""
    res = {}
    for pipelined in (False, 16):
        v = _viewport(scene, pipelined)
        got = []
        v.setCamera(_cam(0))
        v.start(1)
        assert _sample_count(v) == 1
        d = v.diagnostics
        assert d["sample_count"] == 1 and d["last_render_ms"] > 0.0
        v.start(3)  # continues the accumulation in flight
        assert _sample_count(v) == 3
        v.setSettings({"maxBounces": 5})  # a reset while the loop runs
        assert _sample_count(v) == 0
        v.start(1)
        v.setCamera(_cam(4))
        v.start(2)
        got.append(v.readAccumulation())
        d = v.diagnostics
        assert d["sample_count"] == 2 and d["traversal_aborted"] == 0
        got.append(d["rays_primary"])
        res[pipelined] = got
        v.dispose()
    np.testing.assert_allclose(res[16][0], res[False][0], **TOL)
    assert res[16][1] == res[False][1]


def test_pipelined_frames_equal_single_frames_of_a_fresh_viewport(scene):
    """Each frame of a pipelined sequence is the one-frame render of its camera."""
    v = _viewport(scene, True)
    bufs = [v.allocReadbackBuffer() for _ in range(3)]
    for k in range(3):
        v.setCamera(_cam(k))
        v.start(1)
        v.readAccumulationAsync(bufs[k])
    v.readWait()
    v.dispose()
    for k in range(3):
        f = _viewport(scene, False)
        f.setCamera(_cam(k))
        f.start(1)
        np.testing.assert_allclose(bufs[k], f.readAccumulation(), **TOL)
        f.dispose()


@pytest.mark.parametrize("pool", [0, 4000])
@pytest.mark.parametrize("depth", [3, 8, 16])
def test_render_ahead_queue(scene, pool, depth):
    """`depth` accumulations in flight: per frame setCamera, start(1),
    readWaitReady() (frame k - depth + 1's copy is complete) and this frame's
    readAccumulationAsync; each image equals the frame rendered alone.  The
    render calls stop at either iteration parity, so the frames cover both."""
    n = depth + 5
    ref = []
    f = _viewport(scene, False, pool=pool)
    for k in range(n):
        f.setCamera(_cam(k % 7))
        f.start(1)
        ref.append(f.readAccumulation())
    f.dispose()
    v = _viewport(scene, depth, pool=pool)
    bufs = [v.allocReadbackBuffer() for _ in range(n)]
    for k in range(n):
        v.setCamera(_cam(k % 7))
        v.start(1)
        in_flight = v.readWaitReady()
        assert 0 <= in_flight <= depth - 1
        if k >= depth - 1:  # frame k - depth + 1 has finished and its copy is on the host
            np.testing.assert_allclose(bufs[k - depth + 1], ref[k - depth + 1], **TOL)
        v.readAccumulationAsync(bufs[k])
    v.readWait()
    d = v.diagnostics
    assert d["rays_primary"] == n * 96 * 64 and d["traversal_aborted"] == 0
    v.dispose()
    for k in range(n):
        np.testing.assert_allclose(bufs[k], ref[k], **TOL)
