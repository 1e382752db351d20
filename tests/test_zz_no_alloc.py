"""latec_quantize_static -- the quantizer for callers that cannot allocate.

Some callers cannot call cudaMalloc (their device memory belongs to another
allocator, or a cudaMalloc/cudaFree would stall a latency-critical loop by
synchronising the device). For them the library exports latec_quantize_static,
which keeps its scratch in a fixed file-scope device array instead of a
caller-provided workspace. These tests call it through the C ABI and check
that it returns exactly what the workspace entry point latec_quantize returns
(codes, reconstruction, outliers, statistics and histograms, compared bit for
bit as the other quantizer tests do), on two calls in a row so that state left
in the shared scratch by one call cannot leak into the next, and that inputs
beyond its fixed limit are refused with a clear error.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from latec_b200 import _lib

    return _lib, _lib.load()


def _case(n, dtype, seed):
    rs = np.random.RandomState(seed)
    x = (rs.randn(n) * 10.0).astype(dtype)
    pred = (x + rs.randn(n) * 0.02).astype(dtype)
    x[rs.rand(n) < 0.01] = 1e6   # beyond the radius: outliers
    x[::997] = np.nan            # outliers by verification
    return x, pred


def _quantize(entry, x, pred, eb, radius=1 << 15):
    import torch

    L, lib = _lib()
    f64 = x.dtype == np.float64
    dev = torch.device("cuda")
    n = len(x)
    xd = torch.from_numpy(x).to(dev)
    pd = torch.from_numpy(pred).to(dev)
    codes = torch.full((max(n, 1),), -1, dtype=torch.int16, device=dev)
    recon = torch.full((max(n, 1),), 7.0, dtype=xd.dtype, device=dev)
    outl = torch.full((max(n, 1),), 3.0, dtype=xd.dtype, device=dev)
    stats = torch.full((ctypes.sizeof(L.StageStats),), 0xAB, dtype=torch.uint8, device=dev)
    segs = max(1, -(-n // (1 << 22)))
    hseg = torch.full((segs * 512,), 5, dtype=torch.int32, device=dev)
    htot = torch.full((65536,), 5, dtype=torch.int32, device=dev)
    prm = L.QuantParams(dtype=L.F64 if f64 else L.F32, channels=1, radius=radius, order=1,
                        center=0, end_mode=1, round_output=0, reserved=0)
    sp = torch.cuda.current_stream().cuda_stream
    if entry == "workspace":
        ws = torch.empty(int(lib.latec_flat_workspace_bytes(n, prm.dtype)), dtype=torch.uint8,
                         device=dev)
        rc = lib.latec_quantize(ctypes.byref(prm), eb, n, xd.data_ptr(), pd.data_ptr(),
                                codes.data_ptr(), recon.data_ptr(), outl.data_ptr(),
                                stats.data_ptr(), hseg.data_ptr(), htot.data_ptr(), ws.data_ptr(),
                                ws.numel(), sp)
    else:
        rc = lib.latec_quantize_static(ctypes.byref(prm), eb, n, xd.data_ptr(), pd.data_ptr(),
                                       codes.data_ptr(), recon.data_ptr(), outl.data_ptr(),
                                       stats.data_ptr(), hseg.data_ptr(), htot.data_ptr(), sp)
    assert rc == 0, rc
    torch.cuda.synchronize()
    st = L.StageStats.from_buffer_copy(stats.cpu().numpy().tobytes())
    n_out = st.n_out
    return dict(codes=codes[:n].cpu().numpy(), recon=recon[:n].cpu().numpy(),
                outliers=outl[:n_out].cpu().numpy(), n_out=n_out, maxq=st.maxq,
                stats=np.array(st.stats[:]), hseg=hseg.cpu().numpy(), htot=htot.cpu().numpy())


def _same(a, b):
    assert a["n_out"] == b["n_out"] and a["maxq"] == b["maxq"]
    assert np.array_equal(a["codes"], b["codes"])
    assert np.array_equal(a["recon"].view(np.uint8), b["recon"].view(np.uint8))
    assert np.array_equal(a["outliers"].view(np.uint8), b["outliers"].view(np.uint8))
    assert np.array_equal(a["stats"].view(np.uint8), b["stats"].view(np.uint8))
    assert np.array_equal(a["hseg"], b["hseg"]) and np.array_equal(a["htot"], b["htot"])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_static_quantizer_matches_workspace_quantizer_twice(dtype):
    # two calls in a row: a large one with many outliers, then a smaller one
    for n, seed, eb in [(300_000, 1, 0.01), (70_001, 2, 0.05)]:
        x, pred = _case(n, dtype, seed)
        want = _quantize("workspace", x, pred, eb)
        got = _quantize("static", x, pred, eb)
        assert want["n_out"] > 0
        _same(got, want)


def test_static_quantizer_accepts_its_limit_and_refuses_more():
    L, lib = _lib()
    limit = 1 << 19
    x, pred = _case(limit, np.float32, 3)
    _same(_quantize("static", x, pred, 0.01), _quantize("workspace", x, pred, 0.01))
    prm = L.QuantParams(dtype=L.F32, channels=1, radius=1 << 15, order=1, center=0, end_mode=1,
                        round_output=0, reserved=0)
    rc = lib.latec_quantize_static(ctypes.byref(prm), 0.01, limit + 1, 1, 1, 1, 1, 1, 1, 1, 1, 0)
    assert rc == -7  # LATEC_ERR_TOO_LARGE, before any pointer is touched
