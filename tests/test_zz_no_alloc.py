"""The allocation-free table build, for hosts that cannot let this library
allocate device memory (an engine that owns all device memory through its own
pool, or a frame loop that cannot take cudaMalloc's implicit synchronisation).

dspbr_ibl_tables_noalloc is called through the C ABI with buffers the test
allocates itself (torch owns the device memory here), and its tables must equal
those of the allocating entry point, dspbr_ibl_create, bit for bit, on two calls
in a row with different images.  This file is collected last on purpose: it
also runs after every other test has used the library in the same process."""
import numpy as np
import pytest

from dspbr import _lib, synth
from dspbr.viewport import Context, DeviceIbl

pytestmark = pytest.mark.gpu


def _noalloc_tables(torch, env, stream=None):
    """The tables through dspbr_ibl_tables_noalloc.  The inputs are uploaded
    and the outputs allocated on `stream` (torch's current stream if None),
    and the call is ordered on that stream."""
    h, w = env.shape[0], env.shape[1]
    dev = torch.device("cuda", 0)
    stream = stream or torch.cuda.current_stream(dev)
    with torch.cuda.stream(stream):
        rgba = torch.from_numpy(np.ascontiguousarray(env, np.float32)).to(dev, non_blocking=False)
        pdf = torch.full((w * h,), -1.0, dtype=torch.float32, device=dev)
        cdf = torch.full((w * h,), -1.0, dtype=torch.float32, device=dev)
        ypdf = torch.full((h,), -1.0, dtype=torch.float32, device=dev)
        ycdf = torch.full((h,), -1.0, dtype=torch.float32, device=dev)
        total = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
        rc = _lib.load().dspbr_ibl_tables_noalloc(rgba.data_ptr(), w, h, pdf.data_ptr(), cdf.data_ptr(),
                                                  ypdf.data_ptr(), ycdf.data_ptr(), total.data_ptr(),
                                                  stream.cuda_stream)
        assert rc == 0
    stream.synchronize()
    return {"pdf": pdf.cpu().numpy(), "cdf": cdf.cpu().numpy(), "yPdf": ypdf.cpu().numpy(),
            "yCdf": ycdf.cpu().numpy(), "totalSum": float(total.cpu().numpy()[0])}


def _assert_same_tables(got, want):
    for k in ("pdf", "cdf", "yPdf", "yCdf"):
        np.testing.assert_array_equal(got[k].view(np.uint32), want[k].view(np.uint32), err_msg=k)
    assert got["totalSum"] == want["totalSum"]


def test_noalloc_tables_match_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    ctx = Context(0)
    envs = [synth.env_lognormal(512, 256, np.random.default_rng(1)),
            synth.env_sun(256, 128, 0.3, (0.2, 0.9, 0.3), 500.0, 2.0)]
    for env in envs:  # two calls in a row through the shared scratch array
        _assert_same_tables(_noalloc_tables(torch, env), DeviceIbl(ctx, env).tables())
    ctx.close()


def test_noalloc_on_a_caller_stream_and_edge_maps():
    """Ordered on a non-default stream of the caller; a one-texel-wide map
    with an all-black row (row sum 0 -> 1, renderer.ts:786-787); and the
    largest map the scratch array holds, 16384 rows."""
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    ctx = Context(0)
    side = torch.cuda.Stream(device=0)
    narrow = np.random.default_rng(3).uniform(0.0, 2.0, (9, 1, 4)).astype(np.float32)
    narrow[4] = 0.0
    tall = np.random.default_rng(4).uniform(0.0, 1.0, (16384, 2, 4)).astype(np.float32)
    for env in (narrow, tall, synth.env_sun(64, 32, 0.3, (0.2, 0.9, 0.3), 500.0, 6.0)):
        _assert_same_tables(_noalloc_tables(torch, env, stream=side), DeviceIbl(ctx, env).tables())
    ctx.close()


def test_noalloc_refuses_misaligned_buffers():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    buf = torch.zeros(64, dtype=torch.float32, device=dev)
    p = buf.data_ptr()
    lib = _lib.load()
    # rgba32f not 16-byte aligned; total_sum not 8-byte aligned (refused on the host, nothing launched)
    assert lib.dspbr_ibl_tables_noalloc(p + 4, 1, 2, p + 64, p + 128, p + 160, p + 192, p + 224, None) == -1
    assert lib.dspbr_ibl_tables_noalloc(p, 1, 2, p + 64, p + 128, p + 160, p + 192, p + 228, None) == -1


def test_noalloc_refuses_maps_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float32, device=dev)
    rc = _lib.load().dspbr_ibl_tables_noalloc(buf.data_ptr(), 1, 16385, buf.data_ptr(), buf.data_ptr(),
                                              buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None)
    assert rc == -1
