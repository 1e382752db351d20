"""Training kernels of the learned predictor: the gradient of the
teacher-forced stage schedule equals PyTorch autograd on a plain float32
restatement of the network (tests/torch_gnn_ref.py), the rate loss and its
gradient match autograd on every branch, AdamW matches torch.optim.AdamW, and
a short run lowers the loss and yields a checkpoint the codec loads."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _weights_t(w, device):
    import torch

    return {k: torch.tensor(np.asarray(v, np.float32), device=device, requires_grad=True)
            for k, v in w.items()}


@pytest.mark.parametrize("shape,levels,stride,batch", [((16, 16), 2, 4, 2), ((12, 10), 2, 4, 3),
                                                       ((8, 8, 8, 8), 2, 4, 2),
                                                       ((6, 5, 7), 1, 2, 2)],
                         ids=["2d16", "2d12x10", "4d8", "3d"])
def test_gradient_matches_autograd(shape, levels, stride, batch):
    import torch

    from latec_b200 import gnn, synthetic
    from latec_b200.train import Trainer
    from torch_gnn_ref import run_stages_loss

    w = gnn.random_weights(3, 64, 1)
    tr = Trainer(d=64, agg_level=1, weights=w, mse_weight=0.5, ema_decay=0)
    x = synthetic.sample_synthetic_batch(batch, shape, (1.0, 8.0), np.random.default_rng(7),
                                         device="cuda")
    eb = torch.tensor(np.geomspace(1e-3, 2e-2, batch), dtype=torch.float32, device="cuda")
    tr.zero_grad()
    bits, mse, mae, npix = tr.run_stages(x, shape, levels, stride, eb, teacher_noise=False)
    torch.cuda.synchronize()
    got = tr.g.detach().cpu().double().numpy()

    W = _weights_t(w, "cuda")
    loss, ref_bits = run_stages_loss(W, x, tr.geoms(shape, levels, stride), eb, 64, 0.5)
    loss.backward()
    want = np.concatenate([W[k].grad.detach().cpu().double().numpy().reshape(-1)
                           for k in gnn.param_shapes(64, 1)])
    assert math.isclose(bits, float(ref_bits.detach()), rel_tol=1e-4)
    # float32 on both sides, different summation orders
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert rel < 2e-3, rel
    np.testing.assert_allclose(got, want, rtol=5e-2, atol=2e-3 * np.abs(want).max())


def test_loss_and_gradient_on_every_branch():

    import torch

    from latec_b200 import _lib
    from torch_gnn_ref import laplace_bits

    lib = _lib.load()
    rng = np.random.default_rng(0)
    B, M = 4, 4096
    eb = torch.tensor([1e-4, 1e-3, 1e-2, 5e-2], dtype=torch.float32, device="cuda")
    tgt = torch.tensor(rng.uniform(0, 1, (B, M)), dtype=torch.float32, device="cuda")
    # residuals inside the cell, in the tail, and far in the tail (> 32 bits)
    spread = np.concatenate([rng.uniform(-0.5, 0.5, M // 4) * 1e-4,
                             rng.uniform(-1, 1, M // 4) * 1e-2,
                             rng.uniform(-1, 1, M // 4) * 0.3,
                             rng.uniform(-1, 1, M - 3 * (M // 4))])
    mu = (tgt + torch.tensor(spread, dtype=torch.float32, device="cuda")).contiguous()
    lb = torch.tensor(rng.uniform(-18, -2, (B, M)), dtype=torch.float32, device="cuda")
    mw, scale = 0.7, 1.0 / (B * M)
    dmu, dlb = torch.empty_like(mu), torch.empty_like(lb)
    acc = torch.zeros(3, dtype=torch.float64, device="cuda")
    _lib.check(lib.latec_tr_loss(mu.data_ptr(), lb.data_ptr(), tgt.data_ptr(), B * M, M,
                                 eb.data_ptr(), mw, scale, dmu.data_ptr(), dlb.data_ptr(),
                                 acc.data_ptr(), _lib.stream_ptr()))
    m_ = mu.detach().clone().requires_grad_(True)
    l_ = lb.detach().clone().requires_grad_(True)
    bits = laplace_bits(m_, l_, tgt, eb)
    loss = (bits.sum() + mw * ((m_ - tgt) ** 2).sum()) * scale
    loss.backward()
    assert math.isclose(float(acc[0]), float(bits.sum()), rel_tol=1e-5)
    np.testing.assert_allclose(dmu.cpu().numpy(), m_.grad.cpu().numpy(), rtol=2e-3,
                               atol=1e-6 * float(m_.grad.abs().max()))
    np.testing.assert_allclose(dlb.cpu().numpy(), l_.grad.cpu().numpy(), rtol=2e-3,
                               atol=1e-6 * float(l_.grad.abs().max()))


def test_adamw_matches_torch():
    import torch

    from latec_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(1)
    n = 10_000
    p0 = rng.standard_normal(n).astype(np.float32)
    p = torch.tensor(p0, device="cuda")
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    q = torch.tensor(p0, device="cuda", requires_grad=True)
    opt = torch.optim.AdamW([q], lr=2e-3, weight_decay=1e-3)
    for step in range(1, 6):
        g = torch.tensor(rng.standard_normal(n).astype(np.float32), device="cuda")
        _lib.check(lib.latec_tr_adamw(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), n,
                                      2e-3, 0.9, 0.999, 1e-8, 1e-3, step, _lib.stream_ptr()))
        q.grad = g.clone()
        opt.step()
    np.testing.assert_allclose(p.cpu().numpy(), q.detach().cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_short_run_lowers_the_loss_and_saves_a_loadable_checkpoint(tmp_path):
    import torch

    import latec_b200 as lb
    from latec_b200 import fields
    from latec_b200.train import train

    tr, hist = train(40, shape4=(8, 8, 8, 8), batch4=2, shape2=(32, 32), batch2=4, stride4=4,
                     warmup=5, seed=1, log_every=0, device="cuda")
    first = np.mean([h["synthetic"][0] for h in hist[:5]])
    last = np.mean([h["synthetic"][0] for h in hist[-5:]])
    assert np.isfinite(last) and last < first, (first, last)
    path = str(tmp_path / "ckpt.pt")
    tr.save(path)
    codec = lb.GNNCodec(checkpoint_path=path)
    x = fields.mixed_4d((16, 16, 16, 16), seed=2, device="cuda")
    vmin, vmax = float(x.min()), float(x.max())
    span = vmax - vmin
    s = codec.compress(x, 1e-3, levels=3)
    y = torch.as_tensor(codec.uncompress(s), device="cuda")
    # the bound holds on the normalised values; float32 (de)normalisation slack
    slack = 2.0 ** -24 * (3.0 * span + max(abs(vmin), abs(vmax)))
    assert float((y.double() - x.double()).abs().max()) <= 1e-3 * span + slack
