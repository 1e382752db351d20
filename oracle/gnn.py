"""The axial GNN predictor on the CPU in float64 -- TEST INFRASTRUCTURE ONLY.

Restates the reference model (``latec/gnn_predictor.py:593-933`` build_model
with InitEmbed, DirState, DirEmbed, BiDirEmbed, AttnPool, PredHead, MixEmbed)
and one codec stage of it (``:984-1000`` stage_forward) in NumPy float64, and
the neighbour geometry by the exhaustive scan the reference's own geometry is
tested against (``tests/test_gnn_predictor.py:33-73``).

Weights are a dict keyed by the reference's ``state_dict`` names. Pinned to
golden outputs of the reference module itself (``tests/golden/gnn.npz``,
made by ``tests/golden/make_gnn_golden.py``), which runs in float32: the
comparison is within float32 rounding, not bit-exact.
"""

from __future__ import annotations

import itertools

import numpy as np
from scipy.special import erf

from . import levels as olevels


def half_directions(ndim, agg_level=None):
    """``latec/gnn_predictor.py:116-136``."""
    out = []
    for d in itertools.product((-1, 0, 1), repeat=ndim):
        first = next((x for x in d if x != 0), 0)
        if first > 0 and (agg_level is None or sum(x != 0 for x in d) <= agg_level):
            out.append(d)
    return out


# ------------------------------------------------------------------ geometry

def _nearest(known, dvec, limit):
    """Nearest known sample along +dvec within ``limit`` steps: (step, valid)."""
    shape = known.shape
    step = np.zeros(shape, np.int64)
    found = np.zeros(shape, bool)
    idx = np.indices(shape)
    for t in range(1, limit + 1):
        nb = [idx[k] + t * dvec[k] for k in range(len(shape))]
        inb = np.ones(shape, bool)
        for k in range(len(shape)):
            inb &= (nb[k] >= 0) & (nb[k] < shape[k])
        hit = np.zeros(shape, bool)
        sel = inb & ~found
        if sel.any():
            hit[sel] = known[tuple(n[sel] for n in nb)]
        step[hit] = t
        found |= hit
        if found.all():
            break
    return step, found


def stage_geoms(shape, levels, stride, block, max_radius, agg_level=None):
    """Per non-empty stage: query flat indices and, per half-direction line,
    neighbour steps / validity on both sides (``latec/gnn_predictor.py:270-443``
    semantics: step 0 where invalid, neighbours within ``min(max_radius,
    max(shape))`` steps)."""
    shape = tuple(int(n) for n in shape)
    limit = min(int(max_radius), max(shape))
    dirs = half_directions(len(shape), agg_level)
    strides = np.cumprod((1,) + shape[:0:-1])[::-1].astype(np.int64)
    out = []
    known = np.zeros(shape, bool)
    for mask, _s, _axes in olevels.iter_plan(shape, levels, stride, block):
        if mask.any():
            q = np.flatnonzero(mask)
            sp, sn, vp, vn = [], [], [], []
            for d in dirs:
                for side, sd, sl, vl in (("p", d, sp, vp), ("n", tuple(-c for c in d), sn, vn)):
                    st, ok = _nearest(known, sd, limit)
                    sl.append(np.where(ok, st, 0).reshape(-1)[q])
                    vl.append(ok.reshape(-1)[q])
            dv = np.asarray(dirs, np.float64)
            nnz = np.count_nonzero(dv, axis=1).astype(np.float64)
            out.append(dict(
                query_idx=q.astype(np.int64),
                sp=np.stack(sp), sn=np.stack(sn), vp=np.stack(vp), vn=np.stack(vn),
                off=(dv.astype(np.int64) @ strides),
                cos=dv / np.sqrt(nnz)[:, None], lognnz=0.5 * np.log2(nnz)))
        known |= mask
    return out


def lines(g):
    """``latec/gnn_predictor.py:410-443`` lines(): (ip, in_, dp, dn, vp, vn)."""
    q = g["query_idx"][None, :]
    off = g["off"][:, None]
    vp, vn = g["vp"], g["vn"]
    ip = (q + g["sp"] * off) * vp
    in_ = (q - g["sn"] * off) * vn
    dp = np.maximum(g["sp"], 1).astype(np.float64)
    dn = np.maximum(g["sn"], 1).astype(np.float64)
    return ip, in_, dp, dn, vp, vn


# ------------------------------------------------------------------ model

def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def _lin(w, name, x):
    return x @ w[name + ".weight"].T.astype(np.float64) + w[name + ".bias"].astype(np.float64)


def _mlp(w, prefix, x):
    return _lin(w, prefix + ".2", gelu(_lin(w, prefix + ".0", x)))


def dir_state_index(cos, sign, L):
    """``latec/gnn_predictor.py:681-693``."""
    v = sign * np.asarray(cos, np.float32)
    with np.errstate(divide="ignore"):
        nnz = np.round(1.0 / np.square(v.astype(np.float32)))
    idx = np.where(v > 0, 2 * L - nnz + 1, np.where(v < 0, nnz - 1, float(L)))
    return np.clip(idx, 0, 2 * L).astype(np.int64)


def attn_pool(w, prefix, msgs, valid):
    """``latec/gnn_predictor.py:724-749``: msgs (L, N, d), valid (L, N)."""
    d = msgs.shape[-1]
    v = _lin(w, prefix + ".wv", msgs)
    scale = d ** -0.5
    scores = _mlp_seq(w, prefix + ".wk", msgs)[..., 0] * scale
    scores = np.where(valid, scores, -np.inf)
    sn = float(w[prefix + ".null_k"]) * scale
    scores = np.concatenate([scores, np.full((1,) + scores.shape[1:], sn)], 0)
    v = np.concatenate([v, np.broadcast_to(w[prefix + ".null_v"].astype(np.float64),
                                           (1,) + v.shape[1:])], 0)
    mx = scores.max(0, keepdims=True)
    e = np.exp(scores - mx)
    p = e / e.sum(0, keepdims=True)
    return (p[..., None] * v).sum(0)


def _mlp_seq(w, prefix, x):
    # AttnPool.wk is a bare Sequential (Linear, GELU, Linear): keys prefix.0 / prefix.2
    return _lin(w, prefix + ".2", gelu(_lin(w, prefix + ".0", x)))


def embed(w, E, g, agg_level):
    """Per-axis contexts at the stage's queries (``GNN.embed``): E (B, N, K, d)
    -> (B, M, K, d)."""
    B, N, K, d = E.shape
    ip, in_, dp, dn, vp, vn = lines(g)
    L, M = vp.shape
    table = w["dir_state.table"].astype(np.float64)
    cosl = g["cos"]  # (L, K)
    idx_p = dir_state_index(cosl, 1.0, agg_level)  # (L, K)
    idx_n = dir_state_index(cosl, -1.0, agg_level)
    lognnz = g["lognnz"][:, None]
    lp = np.log2(dp) + lognnz
    ln = np.log2(dn) + lognnz
    msgs = np.zeros((B, L, M, K, d))
    for l in range(L):
        ep = np.concatenate([E[:, ip[l]], np.broadcast_to(table[idx_p[l]], (B, M, K, table.shape[1]))], -1)
        en = np.concatenate([E[:, in_[l]], np.broadcast_to(table[idx_n[l]], (B, M, K, table.shape[1]))], -1)
        lpe = np.broadcast_to(lp[l][None, :, None, None], (B, M, K, 1))
        lne = np.broadcast_to(ln[l][None, :, None, None], (B, M, K, 1))
        both = _mlp(w, "bidir.net", np.concatenate([en, ep, lne, lpe], -1))
        pos_only = vp[l] & ~vn[l]
        neg_only = vn[l] & ~vp[l]
        one = np.where(pos_only[None, :, None, None], ep, en)
        sign = np.where(pos_only, 1.0, -1.0)[None, :, None, None] * np.ones((B, M, K, 1))
        lse = np.where(pos_only[None, :, None, None], lpe, lne)
        side = _mlp(w, "dir.net", np.concatenate([one, sign, lse], -1))
        live = vp[l] | vn[l]
        m = np.where((pos_only | neg_only)[None, :, None, None], side, both)
        msgs[:, l] = np.where(live[None, :, None, None], m, 0.0)
    valid = vp | vn  # (L, M)
    flat = msgs.transpose(1, 0, 2, 3, 4).reshape(L, B * M * K, d)
    vflat = np.broadcast_to(valid[:, None, :, None], (L, B, M, K)).reshape(L, B * M * K)
    ctx = attn_pool(w, "line_pool", flat, vflat)
    return ctx.reshape(B, M, K, d)


def finalize(w, ctx, vals):
    """``GNN.finalize``: ctx (B, M, K, d), vals (B, M) -> (B, M, K, d)."""
    ve = _mlp(w, "init.net", np.asarray(vals, np.float64)[..., None])  # (B, M, d)
    ve = np.broadcast_to(ve[:, :, None, :], ctx.shape)
    return _mlp(w, "mix.net", np.concatenate([ctx, ve], -1))


def head_of(w, ctx, eb):
    """``GNN.head_of`` + ``PredHead.forward``: (mu, log_b), each (B, M)."""
    B, M, K, d = ctx.shape
    msgs = ctx.transpose(2, 0, 1, 3).reshape(K, B * M, d)
    pooled = attn_pool(w, "axis_pool", msgs, np.ones((K, B * M), bool)).reshape(B, M, d)
    tiny = float(np.finfo(np.float32).tiny)
    log_eb = np.log2(max(float(eb), tiny))
    out = _mlp(w, "head.net", np.concatenate([pooled, np.full((B, M, 1), log_eb)], -1))
    mu = 1.0 / (1.0 + np.exp(-out[..., 0]))
    log_b = log_eb + np.clip(out[..., 1], -4.0, 12.0)
    return mu, log_b


def stage_forward(w, E, g_prev, g_head, vals, agg_level, finalize_ctx=None, eb=0.01):
    """``latec/gnn_predictor.py:984-1000``: returns ((mu, log_b), E, head_ctx)."""
    if g_prev is not None and len(g_prev["query_idx"]):
        ctx = finalize_ctx if finalize_ctx is not None else embed(w, E, g_prev, agg_level)
        E[:, g_prev["query_idx"]] = finalize(w, ctx, vals)
    head_ctx = embed(w, E, g_head, agg_level)
    return head_of(w, head_ctx, eb), E, head_ctx


def run_stages(w, x, geoms, agg_level, eb=0.01, d=64):
    """Closed loop over every stage of a (B, *S) field whose true values are
    revealed after each stage (the reference tests' loop): per stage (mu, log_b)."""
    B = x.shape[0]
    flat = x.reshape(B, -1).astype(np.float64)
    K = x.ndim - 1
    E = np.zeros((B, flat.shape[1], K, d))
    out, prev, ctx = [], None, None
    for g in geoms:
        vals = flat[:, prev["query_idx"]] if prev is not None else None
        (mu, lb), E, ctx = stage_forward(w, E, prev, g, vals, agg_level, finalize_ctx=ctx, eb=eb)
        out.append((mu, lb))
        prev = g
    return out, E
