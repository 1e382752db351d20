"""Plain PyTorch float32 restatement of the axial GNN forward and of the
training loss, used only as the autograd reference of the training kernels'
gradients (the same model as latec/gnn_predictor.py:593-1000 and
scripts/train_gnn.py:195-241, written on the geometry tensors of
latec_b200.gnn.StageGeom)."""

import math

import torch
import torch.nn.functional as F


def lin(x, W, name):
    return x @ W[name + ".weight"].t() + W[name + ".bias"]


def mlp(x, W, prefix):
    return lin(F.gelu(lin(x, W, prefix + ".0")), W, prefix + ".2")


def embed(W, E, g, d):
    B, N, K, _ = E.shape
    t = g._t
    L, M = g.L, g.M
    np2 = int(g._two_off[1]) if g.struct.n_tiles else 0
    np1 = int(g._one_off[1]) if g.struct.n_tiles else 0
    nbr_p, nbr_n = t["nbr_p"].long().reshape(-1), t["nbr_n"].long().reshape(-1)
    logd_p, logd_n = t["logd_p"].reshape(-1), t["logd_n"].reshape(-1)
    sidx_p, sidx_n = t["sidx_p"].long().reshape(L, K), t["sidx_n"].long().reshape(L, K)
    table = W["dir_state.table"]
    parts = []
    if np2:
        pr = t["two"][:np2].long()
        l = pr // M
        ex = lambda a: a.unsqueeze(0).expand(B, *a.shape)  # noqa: E731
        X = torch.cat([E[:, nbr_n[pr]], ex(table[sidx_n[l]]), E[:, nbr_p[pr]], ex(table[sidx_p[l]]),
                       ex(logd_n[pr][:, None, None].expand(np2, K, 1)),
                       ex(logd_p[pr][:, None, None].expand(np2, K, 1))], -1)
        parts.append(mlp(X, W, "bidir.net"))
    if np1:
        pr = t["one"][:np1].long()
        l = pr // M
        pos = nbr_p[pr] >= 0
        nb = torch.where(pos, nbr_p[pr], nbr_n[pr])
        s = table[torch.where(pos[:, None], sidx_p[l], sidx_n[l])]
        sign = torch.where(pos, 1.0, -1.0).to(E.dtype)[:, None, None].expand(np1, K, 1)
        ld = torch.where(pos, logd_p[pr], logd_n[pr])[:, None, None].expand(np1, K, 1)
        ex = lambda a: a.unsqueeze(0).expand(B, *a.shape)  # noqa: E731
        X = torch.cat([E[:, nb], ex(s), ex(sign), ex(ld)], -1)
        parts.append(mlp(X, W, "dir.net"))
    scale = 1.0 / math.sqrt(d)
    nk = W["line_pool.null_k"] * scale
    nv = W["line_pool.null_v"]
    if not parts:
        return nv.expand(B, M, K, d).clone()
    MS = torch.cat(parts, 1)
    key = lin(F.gelu(lin(MS, W, "line_pool.wk.0")), W, "line_pool.wk.2")[..., 0]
    V = lin(MS, W, "line_pool.wv")
    row_of = t["row_of"].long().reshape(L, M)
    valid = row_of >= 0
    idx = row_of.clamp_min(0)
    kc = key[:, idx] * scale  # (B, L, M, K)
    kc = torch.where(valid[None, :, :, None], kc, torch.full_like(kc, -math.inf))
    sc = torch.cat([kc, nk.reshape(1, 1, 1, 1).expand(B, 1, M, K)], 1)
    p = torch.softmax(sc, 1)
    vc = V[:, idx]  # (B, L, M, K, d)
    ctx = (p[:, :L, :, :, None] * vc).sum(1) + p[:, L:, :, :, None].squeeze(1) * nv
    return ctx


def head(W, ctx, log_eb, d):
    B, M, K, _ = ctx.shape
    scale = 1.0 / math.sqrt(d)
    key = lin(F.gelu(lin(ctx, W, "axis_pool.wk.0")), W, "axis_pool.wk.2")[..., 0] * scale
    V = lin(ctx, W, "axis_pool.wv")
    sc = torch.cat([key, (W["axis_pool.null_k"] * scale).reshape(1, 1, 1).expand(B, M, 1)], -1)
    p = torch.softmax(sc, -1)
    pooled = (p[..., :K, None] * V).sum(2) + p[..., K:] * W["axis_pool.null_v"]
    X = torch.cat([pooled, log_eb[:, None, None].expand(B, M, 1)], -1)
    O = mlp(X, W, "head.net")
    return torch.sigmoid(O[..., 0]), log_eb[:, None] + O[..., 1].clamp(-4.0, 12.0)


def finalize(W, ctx, vals, g, E):
    B, M, K, d = ctx.shape
    VE = mlp(vals[..., None], W, "init.net")
    X = torch.cat([ctx, VE[:, :, None, :].expand(B, M, K, d)], -1)
    Y = mlp(X, W, "mix.net")
    return E.index_copy(1, g._t["query"].long(), Y)


def laplace_bits(mu, log_b, target, eb):
    """discretized_laplace_nll (train_gnn.py:195-232), restated."""
    eb = eb.reshape(-1, 1)
    b = torch.exp2(log_b).clamp_min(torch.finfo(target.dtype).tiny)
    abs_r = (target - mu).abs()
    rho = abs_r / b
    e = eb / b
    tail_mass = torch.log1p(-torch.exp((-2.0 * e).clamp_max(-torch.finfo(target.dtype).eps)))
    t = rho - e
    t_max = 32.0 * math.log(2.0)
    t = torch.where(t > t_max, t_max + torch.log1p((t - t_max).clamp_min(0.0)), t)
    logp_tail = -math.log(2.0) - t + tail_mass
    rc = torch.minimum(rho, e)
    cross = 1.0 - 0.5 * torch.exp(-(e - rc)) - 0.5 * torch.exp(-(e + rc))
    logp_cross = torch.log(cross.clamp_min(1e-30))
    logp = torch.where(abs_r >= eb, logp_tail, logp_cross)
    return -logp / math.log(2.0)


def run_stages_loss(W, x, geoms, eb, d, mse_weight):
    """Teacher-forced (exact truth) closed loop; (bits + mse_weight * sq) / points."""
    B, N = x.shape
    K = geoms[0].K
    E = torch.zeros(B, N, K, d, device=x.device)
    log_eb = torch.log2(eb)
    ctx = embed(W, E, geoms[0], d)
    bits = torch.zeros((), device=x.device)
    sq = torch.zeros((), device=x.device)
    npix = 0
    for i in range(1, len(geoms)):
        gp, gh = geoms[i - 1], geoms[i]
        E = finalize(W, ctx, x[:, gp.query_idx], gp, E)
        ctx = embed(W, E, gh, d)
        mu, lb = head(W, ctx, log_eb, d)
        tgt = x[:, gh.query_idx]
        bits = bits + laplace_bits(mu, lb, tgt, eb).sum()
        sq = sq + ((mu - tgt) ** 2).sum()
        npix += tgt.numel()
    return (bits + mse_weight * sq) / npix, bits / npix
