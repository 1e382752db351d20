"""Mixed-precision training GEMMs: latec_tr_linear_bf16 / _bwd_bf16 round both
operands of every GEMM to BF16 and accumulate in float32 (tcgen05 tensor cores
for tiles at least 32 wide, SIMT tiles for the narrow layers). Each output is
checked against a float64 product of the BF16-rounded operands, and must lie
much closer to it than to the float32 product. A BF16 trainer's gradient stays
close to the float32 trainer's, and a short BF16 run lowers the loss."""

import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SQ2 = math.sqrt(2.0)


def _bf(t):
    import torch

    return t.to(torch.bfloat16).double()


def _gelu(z):
    import torch

    return 0.5 * z * (1.0 + torch.erf(z / SQ2))


def _gelu_d(z):
    import torch

    return 0.5 * (1.0 + torch.erf(z / SQ2)) + z * torch.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def _rel(a, b):
    return float((a - b).norm() / b.norm())


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


CASES = [(1000, 162, 128), (700, 64, 64), (300, 65, 128), (257, 128, 2), (130, 64, 1),
         (20000, 128, 64), (33, 1, 64)]


@pytest.mark.parametrize("rows,fin,fout", CASES)
@pytest.mark.parametrize("act", [0, 1])
def test_linear_forward(rows, fin, fout, act):
    import torch

    from latec_b200 import _lib

    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(rows + fin + fout + act)
    X = torch.randn(rows, fin, device="cuda", generator=g)
    W = torch.randn(fout, fin, device="cuda", generator=g) / math.sqrt(fin)
    b = torch.randn(fout, device="cuda", generator=g)
    Y = torch.full((rows, fout), float("nan"), device="cuda")
    Z = torch.full((rows, fout), float("nan"), device="cuda") if act else None
    _lib.check(lib.latec_tr_linear_bf16(_ptr(X), fin, rows, fin, _ptr(W), _ptr(b), fout, _ptr(Y),
                                        fout, act, _ptr(Z), _lib.stream_ptr()), "linear_bf16")
    _lib.check(lib.latec_tr_gemm_status(_lib.stream_ptr()), "gemm_status")
    zb = _bf(X) @ _bf(W).T + b.double()
    z32 = X.double() @ W.double().T + b.double()
    want, want32 = (_gelu(zb), _gelu(z32)) if act else (zb, z32)
    got = Y.double()
    assert torch.isfinite(got).all()
    rel = _rel(got, want)
    assert rel < 2e-5, rel
    if fin > 1:  # the operands really were rounded: far closer to the BF16 product
        assert rel * 20 < _rel(got, want32), (rel, _rel(got, want32))
    if act:
        assert _rel(Z.double(), zb) < 2e-5


@pytest.mark.parametrize("rows,fin,fout", CASES)
@pytest.mark.parametrize("act,accum", [(0, 0), (1, 0), (1, 1)])
def test_linear_backward(rows, fin, fout, act, accum):
    import torch

    from latec_b200 import _lib

    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(7 * rows + fin + fout + act)
    X = torch.randn(rows, fin, device="cuda", generator=g)
    W = torch.randn(fout, fin, device="cuda", generator=g) / math.sqrt(fin)
    dY = torch.randn(rows, fout, device="cuda", generator=g)
    Z = torch.randn(rows, fout, device="cuda", generator=g) if act else None
    dX0 = torch.randn(rows, fin, device="cuda", generator=g)
    dX = dX0.clone()
    dW0 = torch.randn(fout, fin, device="cuda", generator=g)
    db0 = torch.randn(fout, device="cuda", generator=g)
    dW, db = dW0.clone(), db0.clone()
    _lib.check(lib.latec_tr_linear_bwd_bf16(_ptr(X), fin, rows, fin, _ptr(W), fout, _ptr(dY),
                                            fout, _ptr(Z), act, _ptr(dX), fin, accum, _ptr(dW),
                                            _ptr(db), _lib.stream_ptr()), "linear_bwd_bf16")
    _lib.check(lib.latec_tr_gemm_status(_lib.stream_ptr()), "gemm_status")
    # dZ is formed in float32 by the kernel before its rounding; the float64
    # restatement can round a handful of its elements the other way, which the
    # relative tolerance absorbs
    dZ = (dY.double() * _gelu_d(Z.double())).float() if act else dY
    dXw = _bf(dZ) @ _bf(W) + (dX0.double() if accum else 0.0)
    dWw = dW0.double() + _bf(dZ).T @ _bf(X)
    dbw = db0.double() + dZ.double().sum(0)
    dX32 = dZ.double() @ W.double() + (dX0.double() if accum else 0.0)
    dW32 = dW0.double() + dZ.double().T @ X.double()
    rx, rw = _rel(dX.double() - (dX0.double() if accum else 0.0),
                  dXw - (dX0.double() if accum else 0.0)), _rel(dW.double() - dW0.double(),
                                                                dWw - dW0.double())
    assert rx < 1e-4, rx
    assert rw < 1e-4, rw
    if fout > 1:
        assert rx * 10 < _rel(dX.double() - (dX0.double() if accum else 0.0),
                              dX32 - (dX0.double() if accum else 0.0))
    if fin > 1:
        assert rw * 10 < _rel(dW.double() - dW0.double(), dW32 - dW0.double())
    np.testing.assert_allclose(db.double().cpu().numpy(), dbw.cpu().numpy(), rtol=1e-4,
                               atol=1e-3 * math.sqrt(rows))


@pytest.mark.parametrize("shape,levels,stride,batch", [((16, 16), 2, 4, 2),
                                                       ((8, 8, 8, 8), 2, 4, 2)],
                         ids=["2d16", "4d8"])
def test_bf16_gradient_close_to_fp32(shape, levels, stride, batch):
    import torch

    from latec_b200 import gnn, synthetic
    from latec_b200.train import Trainer

    w = gnn.random_weights(3, 64, 1)
    x = synthetic.sample_synthetic_batch(batch, shape, (1.0, 8.0), np.random.default_rng(7),
                                         device="cuda")
    eb = torch.tensor(np.geomspace(1e-3, 2e-2, batch), dtype=torch.float32, device="cuda")
    out = {}
    for prec in ("fp32", "bf16"):
        tr = Trainer(d=64, agg_level=1, weights=w, mse_weight=0.5, ema_decay=0, precision=prec)
        tr.zero_grad()
        bits, _, _, _ = tr.run_stages(x, shape, levels, stride, eb, teacher_noise=False)
        torch.cuda.synchronize()
        out[prec] = (bits, tr.g.detach().double().cpu().numpy())
    assert math.isclose(out["bf16"][0], out["fp32"][0], rel_tol=2e-2)
    rel = np.linalg.norm(out["bf16"][1] - out["fp32"][1]) / np.linalg.norm(out["fp32"][1])
    assert rel < 5e-2, rel


def test_bf16_short_run_lowers_the_loss():
    from latec_b200.train import train

    tr, hist = train(40, shape4=(8, 8, 8, 8), batch4=2, shape2=(32, 32), batch2=4, stride4=4,
                     warmup=5, seed=1, log_every=0, device="cuda", precision="bf16")
    first = np.mean([h["synthetic"][0] for h in hist[:5]])
    last = np.mean([h["synthetic"][0] for h in hist[-5:]])
    assert np.isfinite(last) and last < first, (first, last)
    assert tr.skipped_steps == 0
