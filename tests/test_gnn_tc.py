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
