"""The tensor-core (tcgen05, BF16 operands, FP32 accumulation) two-layer MLP
of the GNN message pass against a float64 evaluation of the same BF16-rounded
operands."""

import numpy as np
import pytest
from scipy.special import erf


def _bf16(a):
    """Round float32 to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def _pack(lib, w, kp):
    from latec_b200 import _lib

    n, k = w.shape
    out = np.empty(n * kp, np.uint16)
    w = np.ascontiguousarray(w, np.float32)
    _lib.check(lib.latec_gnn_pack_bf16(w.ctypes.data, n, k, kp, out.ctypes.data))
    return out


def test_pack_layout_on_host():
    """Element (r, c) lands at ((c/8)*(n/8) + r/8)*64 + (r%8)*8 + c%8, padded with zeros."""
    from latec_b200 import _lib

    lib = _lib.load(require_gpu=False)
    n, k, kp = 16, 20, 32
    w = (np.arange(n * k, dtype=np.float32).reshape(n, k) + 1) / 256.0
    p = _pack(lib, w, kp)
    got = np.zeros((n, kp))
    for r in range(n):
        for c in range(kp):
            off = ((c // 8) * (n // 8) + r // 8) * 64 + (r % 8) * 8 + c % 8
            got[r, c] = np.uint32(int(p[off]) << 16).view(np.float32)
    want = np.zeros((n, kp))
    want[:, :k] = _bf16(w)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("pad", [3, None])  # odd row stride (scalar loads) / 16-byte rows
@pytest.mark.parametrize("rows,k1", [(1000, 162), (128, 82), (300, 128), (1, 162), (0, 82)])
def test_mlp2_bf16_matches_float64(rows, k1, pad):
    import torch

    from latec_b200 import _lib

    lib = _lib.load()
    rs = np.random.RandomState(rows + k1)
    k1p = -(-k1 // 16) * 16
    ldx = k1 + 3 if pad else (k1 + 3) // 4 * 4
    X = rs.randn(max(rows, 1), ldx).astype(np.float32)
    W1 = rs.uniform(-1, 1, (128, k1)).astype(np.float32) / np.sqrt(k1)
    b1 = rs.uniform(-0.1, 0.1, 128).astype(np.float32)
    W2 = rs.uniform(-1, 1, (64, 128)).astype(np.float32) / np.sqrt(128)
    b2 = rs.uniform(-0.1, 0.1, 64).astype(np.float32)
    dev = torch.device("cuda")
    xd = torch.from_numpy(X).to(dev)
    w1p = torch.from_numpy(_pack(lib, W1, k1p).view(np.int16)).to(dev)
    w2p = torch.from_numpy(_pack(lib, W2, 128).view(np.int16)).to(dev)
    b1d, b2d = torch.from_numpy(b1).to(dev), torch.from_numpy(b2).to(dev)
    Y = torch.full((max(rows, 1), 70), 9.0, dtype=torch.float32, device=dev)  # ldy 70
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.latec_gnn_mlp2_bf16(xd.data_ptr(), ldx, rows, k1, k1p, w1p.data_ptr(),
                                       b1d.data_ptr(), w2p.data_ptr(), b2d.data_ptr(),
                                       Y.data_ptr(), 70, err.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    y = Y.cpu().numpy()
    if rows == 0:
        assert np.all(y == 9.0)
        return
    H = _gelu(_bf16(X[:, :k1]) @ _bf16(W1).T + b1)
    ref = _bf16(H.astype(np.float32)) @ _bf16(W2).T + b2
    assert np.abs(y[:rows, :64] - ref).max() < 2e-3
    assert np.all(y[:rows, 64:] == 9.0)  # columns beyond the output untouched


# ---------------------------------------------------------------- FP8 (E4M3)
def _e4m3(a):
    """Round float32 values (|v| <= 448) to E4M3, returned as float64."""
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a, np.float32))
    return t.to(torch.float8_e4m3fn).to(torch.float64).numpy()


def _pack8(lib, w, kp):
    from latec_b200 import _lib

    n, k = w.shape
    out = np.empty(n * kp, np.uint8)
    sc = np.empty(n, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    _lib.check(lib.latec_gnn_pack_fp8(w.ctypes.data, n, k, kp, out.ctypes.data, sc.ctypes.data))
    return out, sc


def _unpack8(p, n, kp):
    """Canonical byte (r, c) at ((c/16)*(n/8) + r/8)*128 + (r%8)*16 + c%16."""
    import torch

    r = np.arange(n)[:, None]
    c = np.arange(kp)[None, :]
    off = ((c // 16) * (n // 8) + r // 8) * 128 + (r % 8) * 16 + c % 16
    b = torch.from_numpy(np.ascontiguousarray(p[off]))
    return b.view(torch.float8_e4m3fn).to(torch.float64).numpy()


def test_pack_fp8_layout_on_host():
    from latec_b200 import _lib

    lib = _lib.load(require_gpu=False)
    n, k, kp = 16, 40, 64
    rs = np.random.RandomState(2)
    w = rs.uniform(-3, 3, (n, k)).astype(np.float32)
    w[5] = 0.0  # a zero row keeps scale 1
    p, sc = _pack8(lib, w, kp)
    want_sc = np.where(np.abs(w).max(1) > 0, np.abs(w).max(1) / np.float32(448.0), 1.0)
    np.testing.assert_allclose(sc, want_sc.astype(np.float32), rtol=0)
    got = _unpack8(p, n, kp)
    want = np.zeros((n, kp))
    want[:, :k] = _e4m3(w / sc[:, None])
    assert np.array_equal(got, want)
    assert np.abs(got).max() <= 448.0


def _mlp_fp8_reference(X, k1, W1q, s1, b1, W2q, s2, b2):
    """float64 evaluation of the FP8 kernel's arithmetic on its rounded operands."""
    x = X[:, :k1].astype(np.float32)
    m = np.abs(x).max(1)
    sa = np.where(m > 0, m / np.float32(448.0), np.float32(1.0)).astype(np.float32)
    aq = _e4m3(x * (np.float32(1.0) / sa)[:, None])
    acc1 = aq @ W1q[:, :k1].T
    pre = ((acc1.astype(np.float32) * sa[:, None]) * s1[None, :]).astype(np.float32) + b1
    h = _gelu(pre.astype(np.float64)).astype(np.float32)
    mh = np.abs(h).max(1)
    sh = np.where(mh > 0, mh / np.float32(448.0), np.float32(1.0)).astype(np.float32)
    hq = _e4m3(h * (np.float32(1.0) / sh)[:, None])
    acc2 = hq @ W2q.T
    return (acc2 * sh[:, None]) * s2[None, :] + b2


@pytest.mark.gpu
@pytest.mark.parametrize("rows,k1", [(1000, 162), (128, 82), (300, 128), (1, 162), (0, 82)])
def test_mlp2_fp8_matches_its_float64_emulation(rows, k1):
    import torch

    from latec_b200 import _lib

    lib = _lib.load()
    rs = np.random.RandomState(rows + 2 * k1)
    k1p = -(-k1 // 32) * 32
    ldx = (k1 + 3) // 4 * 4
    X = rs.randn(max(rows, 1), ldx).astype(np.float32)
    W1 = (rs.uniform(-1, 1, (128, k1)) / np.sqrt(k1)).astype(np.float32)
    b1 = rs.uniform(-0.1, 0.1, 128).astype(np.float32)
    W2 = (rs.uniform(-1, 1, (64, 128)) / np.sqrt(128)).astype(np.float32)
    b2 = rs.uniform(-0.1, 0.1, 64).astype(np.float32)
    p1, s1 = _pack8(lib, W1, k1p)
    p2, s2 = _pack8(lib, W2, 128)
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    xd, w1d, s1d, b1d, w2d, s2d, b2d = t(X), t(p1), t(s1), t(b1), t(p2), t(s2), t(b2)
    Y = torch.full((max(rows, 1), 70), 9.0, dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.latec_gnn_mlp2_fp8(xd.data_ptr(), ldx, rows, k1, k1p, w1d.data_ptr(),
                                      s1d.data_ptr(), b1d.data_ptr(), w2d.data_ptr(),
                                      s2d.data_ptr(), b2d.data_ptr(), Y.data_ptr(), 70,
                                      err.data_ptr(), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    y = Y.cpu().numpy()
    if rows == 0:
        assert np.all(y == 9.0)
        return
    want = _mlp_fp8_reference(X, k1, _unpack8(p1, 128, k1p), s1, b1, _unpack8(p2, 64, 128), s2, b2)
    got = y[:rows, :64].astype(np.float64)
    assert np.all(y[:rows, 64:] == 9.0)  # ldy padding untouched
    # float32 accumulation vs float64 may move a hidden value across an E4M3
    # rounding boundary now and then; the bulk agrees closely
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert rel < 1e-2, rel
    exact = _gelu(X[:rows, :k1].astype(np.float64) @ W1.T.astype(np.float64) + b1) @ W2.T + b2
    rel_q = np.linalg.norm(got - exact) / np.linalg.norm(exact)
    assert rel_q < 0.1, rel_q  # E4M3's 3-bit mantissa
