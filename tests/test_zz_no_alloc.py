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


def _noalloc_tables(torch, env):
    h, w = env.shape[0], env.shape[1]
    dev = torch.device("cuda", 0)
    rgba = torch.from_numpy(np.ascontiguousarray(env, np.float32)).to(dev)
    pdf = torch.empty(w * h, dtype=torch.float32, device=dev)
    cdf = torch.empty(w * h, dtype=torch.float32, device=dev)
    ypdf = torch.empty(h, dtype=torch.float32, device=dev)
    ycdf = torch.empty(h, dtype=torch.float32, device=dev)
    total = torch.empty(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = _lib.load().dspbr_ibl_tables_noalloc(rgba.data_ptr(), w, h, pdf.data_ptr(), cdf.data_ptr(), ypdf.data_ptr(),
                                              ycdf.data_ptr(), total.data_ptr(), stream.cuda_stream)
    assert rc == 0
    torch.cuda.synchronize(dev)
    return {"pdf": pdf.cpu().numpy(), "cdf": cdf.cpu().numpy(), "yPdf": ypdf.cpu().numpy(),
            "yCdf": ycdf.cpu().numpy(), "totalSum": float(total.cpu().numpy()[0])}


def test_noalloc_tables_match_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    ctx = Context(0)
    envs = [synth.env_lognormal(512, 256, np.random.default_rng(1)),
            synth.env_sun(256, 128, 0.3, (0.2, 0.9, 0.3), 500.0, 2.0)]
    for env in envs:  # two calls in a row through the shared scratch array
        got = _noalloc_tables(torch, env)
        want = DeviceIbl(ctx, env).tables()
        for k in ("pdf", "cdf", "yPdf", "yCdf"):
            np.testing.assert_array_equal(got[k].view(np.uint32), want[k].view(np.uint32), err_msg=k)
        assert got["totalSum"] == want["totalSum"]
    ctx.close()


def test_noalloc_refuses_maps_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float32, device=dev)
    rc = _lib.load().dspbr_ibl_tables_noalloc(buf.data_ptr(), 1, 16385, buf.data_ptr(), buf.data_ptr(),
                                              buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None)
    assert rc == -1
