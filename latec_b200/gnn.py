"""The axial GNN predictor of the learned LATEC path, evaluated by CUDA
kernels (``latec/gnn_predictor.py``).

Model (``latec/gnn_predictor.py:593-933`` build_model): every point stores one
d-wide embedding per lattice axis. For a query point and each line through
it (the ``half_directions`` of the aggregation level), the nearest known
neighbour on each side is found; a two-sided pair becomes a BiDirEmbed
message, a one-sided one a DirEmbed message, each reading the neighbour's
per-axis embedding concatenated with a learned direction-state vector. The
per-line messages are pooled per axis with single-query attention
(AttnPool), the axes are pooled again, and PredHead reads out a Laplacian
(mu, log2 b) conditioned on log2 eb. Once a point's value is revealed, its
embeddings are finalised by MixEmbed(context, InitEmbed(value)).

Host side here: the weights (a reference checkpoint or seeded random
initialisation with the same names and shapes), the neighbour geometry of
each stage (closed form on the schedule's periodic known-pattern, as the
reference computes it) and the stage loop. Every model evaluation runs in the
kernels of ``csrc/gnn_kernels.cu``: float32 with float32 accumulation in a
fixed order, so the encoder and the decoder predict identically.
"""

from __future__ import annotations

import itertools
import math

import numpy as np

CKPT_VERSION = 7


def _torch():
    import torch

    return torch


# ------------------------------------------------------------------ weights

def param_shapes(d: int = 64, agg_level: int = 1) -> dict:
    """Names and shapes of the model parameters (the reference state_dict)."""
    h, ds = 2 * d, max(1, d // 4)
    de = d + ds
    n_states = 2 * int(agg_level) + 1
    shapes = {}

    def mlp(prefix, sizes):
        for k, (a, b) in enumerate(zip(sizes[:-1], sizes[1:])):
            shapes[f"{prefix}.{2 * k}.weight"] = (b, a)
            shapes[f"{prefix}.{2 * k}.bias"] = (b,)

    mlp("init.net", [1, d, d])
    shapes["dir_state.table"] = (n_states, ds)
    mlp("dir.net", [de + 2, h, d])
    mlp("bidir.net", [2 * de + 2, h, d])
    for pool in ("line_pool", "axis_pool"):
        mlp(f"{pool}.wk", [d, d, 1])
        shapes[f"{pool}.wv.weight"] = (d, d)
        shapes[f"{pool}.wv.bias"] = (d,)
        shapes[f"{pool}.null_k"] = ()
        shapes[f"{pool}.null_v"] = (d,)
    mlp("head.net", [d + 1, h, 2])
    mlp("mix.net", [2 * d, h, d])
    return shapes


def random_weights(seed: int = 0, d: int = 64, agg_level: int = 1) -> dict:
    """Seeded initialisation with the reference's layer scales: Linear layers
    uniform in +-1/sqrt(fan_in), the direction-state table and the null key
    normal scaled by 1/sqrt(width), the null value small normal, and the
    head's log-scale bias at 8 (the reference's "unconfident" start)."""
    rs = np.random.RandomState(seed)
    out = {}
    for name, shp in param_shapes(d, agg_level).items():
        if name.endswith(".weight"):
            bound = 1.0 / math.sqrt(shp[1])
            out[name] = rs.uniform(-bound, bound, shp).astype(np.float32)
        elif name.endswith(".bias"):
            wshape = param_shapes(d, agg_level)[name[:-5] + ".weight"]
            bound = 1.0 / math.sqrt(wshape[1])
            out[name] = rs.uniform(-bound, bound, shp).astype(np.float32)
        elif name == "dir_state.table":
            out[name] = (rs.randn(*shp) * shp[1] ** -0.5).astype(np.float32)
        elif name.endswith("null_k"):
            out[name] = np.float32(rs.randn() * d ** -0.5)
        elif name.endswith("null_v"):
            out[name] = (rs.randn(*shp) * 0.1).astype(np.float32)
    out["head.net.2.bias"][1] = 8.0
    return out


def load_checkpoint(path) -> tuple[dict, int, int]:
    """``latec/gnn_predictor.py:945-981``: (weights, d, agg_level) from a v7
    checkpoint file."""
    torch = _torch()
    ckpt = torch.load(path, map_location="cpu", weights_only=True)
    if int(ckpt.get("version", 1)) != CKPT_VERSION:
        raise ValueError("Axial GNN checkpoint format v7 is required. Retrain with "
                         "scripts/train_gnn.py.")
    if "agg_level" not in ckpt:
        raise ValueError("checkpoint is missing 'agg_level'; retrain with scripts/train_gnn.py.")
    d, agg = int(ckpt["d"]), int(ckpt["agg_level"])
    w = {k: v.detach().cpu().float().numpy() for k, v in ckpt["state_dict"].items()}
    want = param_shapes(d, agg)
    if set(w) != set(want) or any(tuple(w[k].shape) != want[k] for k in want):
        raise ValueError("checkpoint parameters do not match the axial GNN layout")
    return w, d, agg


# ------------------------------------------------------------------ geometry

def half_directions(ndim: int, agg_level: int | None = None) -> list:
    """One offset per line (first non-zero component +1), at most
    ``agg_level`` non-zero components (``latec/gnn_predictor.py:116-136``)."""
    dirs = []
    for d in itertools.product((-1, 0, 1), repeat=ndim):
        first = next((x for x in d if x != 0), 0)
        if first > 0 and (agg_level is None or sum(x != 0 for x in d) <= agg_level):
            dirs.append(d)
    return dirs


def _period_patterns(ndim, levels, stride, block):
    """Known-before-stage pattern of every stage on one period tile
    (``stride`` per axis): each stage of the schedule is a residue condition
    modulo a divisor of the anchor stride, so the field's known mask is the
    tile repeated (the reference's ``_period_prefixes``,
    ``latec/gnn_predictor.py:506-532``)."""
    import ctypes

    from . import _lib
    from .levels import plan_for

    tile = (int(stride),) * ndim
    plan = plan_for(tile, levels, stride, block)
    lib = _lib.load(require_gpu=False)
    pats, cum = [], np.zeros(int(np.prod(tile)), bool)
    for t, n in enumerate(plan.counts):
        pats.append(cum.reshape(tile).copy())
        if n:
            flat = np.empty(n, np.int64)
            _lib.check(lib.latec_plan_stage_flat(plan.handle, t, 0, n, flat.ctypes.data_as(ctypes.c_void_p)))
            cum[flat] = True
    return pats


def _nearest_steps(pat, sd, P, res):
    """Smallest t in [1, P] with pat[(res + t sd) mod P] set, else 0: the hits
    along a lattice line repeat with period P. Points leave the sweep once hit."""
    M = len(res[0])
    step = np.zeros(M, np.int64)
    live = np.arange(M)
    r = [np.asarray(x, np.int64) for x in res]
    for t in range(1, P + 1):
        hit = pat[tuple((r[k] + t * sd[k]) % P for k in range(len(r)))]
        if hit.any():
            step[live[hit]] = t
            keep = ~hit
            live = live[keep]
            r = [x[keep] for x in r]
            if live.size == 0:
                break
    return step


def _state_index(cos, sign, agg_level):
    """DirState row of a signed direction cosine (``latec/gnn_predictor.py:681-693``)."""
    v = np.float32(sign) * np.asarray(cos, np.float32)
    with np.errstate(divide="ignore"):
        nnz = np.round(np.float32(1.0) / np.square(v))
    idx = np.where(v > 0, 2 * agg_level - nnz + 1, np.where(v < 0, nnz - 1, float(agg_level)))
    return np.clip(idx, 0, 2 * agg_level).astype(np.int32)


class StageGeom:
    """Neighbour geometry of one stage (``_StageGeom``, latec/gnn_predictor.py:
    245-443): the query points, and per line the nearest known neighbour on
    each side (flat index or -1) with its log2 distance, plus the live-pair
    lists of each query tile that the message kernels read."""

    def __init__(self, shape, q, pat, P, max_radius, dirs, agg_level, device, m_tile):
        import ctypes

        torch = _torch()
        from . import _lib

        ndim = len(shape)
        shp = np.asarray(shape, np.int64)
        limit = min(int(max_radius), int(shp.max()))
        strides = np.cumprod((1,) + tuple(shape)[:0:-1])[::-1].astype(np.int64)
        self.M, self.L, self.K, self.ndim = len(q), len(dirs), ndim, ndim
        coords = np.stack(np.unravel_index(q, shape), 1).astype(np.int64) if len(q) else \
            np.zeros((0, ndim), np.int64)
        res = tuple(coords[:, k] % P for k in range(ndim))
        nbr = {"p": [], "n": []}
        logd = {"p": [], "n": []}
        steps = {"p": [], "n": []}
        dv = np.asarray(dirs, np.int64)
        nnz = np.count_nonzero(dv, axis=1)
        lognnz = 0.5 * np.log2(nnz.astype(np.float64))
        for l, d in enumerate(dirs):
            for side, sd in (("p", dv[l]), ("n", -dv[l])):
                step = _nearest_steps(pat, sd, P, res) if len(q) else np.zeros(0, np.int64)
                nb = coords + step[:, None] * sd[None, :]
                ok = (step >= 1) & (step <= limit)
                for k in range(ndim):
                    if sd[k] > 0:
                        ok &= nb[:, k] < shp[k]
                    elif sd[k] < 0:
                        ok &= nb[:, k] >= 0
                nbr[side].append(np.where(ok, nb @ strides, -1))
                steps[side].append(np.where(ok, step, 0))
                dist = np.where(ok, step, 1).astype(np.float64)
                logd[side].append((np.log2(dist) + lognnz[l]).astype(np.float32))
        self.query_idx_np = np.asarray(q, np.int64)
        nbr_p, nbr_n = np.stack(nbr["p"]), np.stack(nbr["n"])  # (L, M)
        self.sp, self.sn = np.stack(steps["p"]), np.stack(steps["n"])  # host, 0 = none
        self.valid_p, self.valid_n = nbr_p >= 0, nbr_n >= 0
        cos = (dv / np.sqrt(nnz)[:, None]).astype(np.float32)
        sidx_p = _state_index(cos, 1.0, agg_level)
        sidx_n = _state_index(cos, -1.0, agg_level)
        # live pairs per query tile: two-sided then one-sided, tile-local rows
        self.m_tile = int(m_tile)
        n_tiles = -(-self.M // self.m_tile) if self.M else 0
        two_l, one_l, two_off, one_off = [], [], [0], [0]
        row_of = np.full((self.L, self.M), -1, np.int32)
        both = self.valid_p & self.valid_n
        side = self.valid_p ^ self.valid_n
        for t in range(n_tiles):
            m0, m1 = t * self.m_tile, min(self.M, (t + 1) * self.m_tile)
            l2, mm2 = np.nonzero(both[:, m0:m1])
            l1, mm1 = np.nonzero(side[:, m0:m1])
            p2 = (l2 * self.M + m0 + mm2).astype(np.int32)
            p1 = (l1 * self.M + m0 + mm1).astype(np.int32)
            row_of[l2, m0 + mm2] = np.arange(len(p2), dtype=np.int32)
            row_of[l1, m0 + mm1] = len(p2) + np.arange(len(p1), dtype=np.int32)
            two_l.append(p2)
            one_l.append(p1)
            two_off.append(two_off[-1] + len(p2))
            one_off.append(one_off[-1] + len(p1))

        def dev_i32(a):
            a = np.ascontiguousarray(a, np.int32)
            return torch.from_numpy(a if a.size else np.zeros(1, np.int32)).to(device)

        def dev_f32(a):
            a = np.ascontiguousarray(a, np.float32)
            return torch.from_numpy(a if a.size else np.zeros(1, np.float32)).to(device)

        self._t = dict(
            query=dev_i32(self.query_idx_np), nbr_p=dev_i32(nbr_p), nbr_n=dev_i32(nbr_n),
            logd_p=dev_f32(np.stack(logd["p"])), logd_n=dev_f32(np.stack(logd["n"])),
            two=dev_i32(np.concatenate(two_l) if two_l else np.zeros(0)),
            one=dev_i32(np.concatenate(one_l) if one_l else np.zeros(0)),
            row_of=dev_i32(row_of), sidx_p=dev_i32(sidx_p), sidx_n=dev_i32(sidx_n))
        self._two_off = (ctypes.c_int64 * len(two_off))(*two_off)
        self._one_off = (ctypes.c_int64 * len(one_off))(*one_off)
        g = _lib.GnnGeom()
        g.M, g.L, g.K, g.m_tile, g.n_tiles = self.M, self.L, self.K, self.m_tile, n_tiles
        for name in ("query", "nbr_p", "nbr_n", "logd_p", "logd_n", "two", "one", "row_of",
                     "sidx_p", "sidx_n"):
            setattr(g, name, self._t[name].data_ptr())
        g.two_off = ctypes.cast(self._two_off, ctypes.c_void_p).value
        g.one_off = ctypes.cast(self._one_off, ctypes.c_void_p).value
        self.struct = g
        self.query_idx = self._t["query"].long()


def build_stage_geoms(shape, levels, stride, block, max_radius, agg_level=1, *, device=None,
                      m_tile=1 << 16):
    """Per non-empty stage ``StageGeom`` plus the ``|known| -> index`` map
    (``latec/gnn_predictor.py:535-580``)."""
    import ctypes

    from . import _lib
    from .levels import plan_for

    torch = _torch()
    dev = torch.device(device) if device is not None else torch.device("cuda")
    shape = tuple(int(n) for n in shape)
    plan = plan_for(shape, levels, stride, block)
    pats = _period_patterns(len(shape), levels, stride, block)
    dirs = half_directions(len(shape), agg_level)
    lib = _lib.load(require_gpu=False)
    geoms, count_to_i, cum = [], {}, 0
    for t, n in enumerate(plan.counts):
        if n:
            q = np.empty(n, np.int64)
            _lib.check(lib.latec_plan_stage_flat(plan.handle, t, 0, n, q.ctypes.data_as(ctypes.c_void_p)))
            count_to_i[cum] = len(geoms)
            geoms.append(StageGeom(shape, q, pats[t], int(stride), max_radius, dirs, agg_level,
                                   dev, m_tile))
        cum += n
    return geoms, count_to_i


# ------------------------------------------------------------------ model

class GNNModel:
    """The axial GNN with its parameters packed on the device in the
    reference state_dict order; every method runs the CUDA kernels."""

    def __init__(self, weights: dict, d: int = 64, agg_level: int = 1, device=None,
                 precision: str = "f32"):
        """``precision``: "f32" (every layer in float32), "bf16" (the
        BiDirEmbed, DirEmbed and MixEmbed MLPs, the line pool's key MLP and
        value projection in BF16 on the tensor cores with float32
        accumulation; the pools' softmax, the axis pool and the readout stay
        float32; d = 64) or "fp8"
        (those MLPs in E4M3 with per-output-channel weight scales and per-row
        activation scales, float32 accumulation; d = 64)."""
        import ctypes

        torch = _torch()
        from . import _lib

        lib = _lib.load()
        if precision not in ("f32", "bf16", "fp8"):
            raise ValueError("precision must be 'f32', 'bf16' or 'fp8'")
        if precision in ("bf16", "fp8") and int(d) != 64:
            raise NotImplementedError("the tensor-core message pass is built for d = 64")
        self.precision = precision
        self.d, self.agg_level = int(d), int(agg_level)
        shapes = param_shapes(self.d, self.agg_level)
        flat = np.concatenate([np.asarray(weights[k], np.float32).reshape(-1) for k in shapes])
        want = int(lib.latec_gnn_param_count(self.d, self.agg_level))
        if flat.size != want:
            raise ValueError(f"GNN parameters: {flat.size} floats, the kernels expect {want}")
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.params = torch.from_numpy(flat).to(self.device)
        m = _lib.GnnModel()
        m.d, m.agg_level, m.params = self.d, self.agg_level, self.params.data_ptr()
        self.tc_err = torch.zeros(1, dtype=torch.int32, device=self.device)
        if precision == "bf16":
            parts = []
            for name in ("bidir.net.0", "bidir.net.2", "dir.net.0", "dir.net.2", "mix.net.0",
                         "mix.net.2"):
                w = np.ascontiguousarray(weights[name + ".weight"], np.float32)
                n, k = w.shape
                kp = -(-k // 16) * 16
                out = np.empty(n * kp, np.uint16)
                _lib.check(lib.latec_gnn_pack_bf16(w.ctypes.data, n, k, kp, out.ctypes.data),
                           "latec_gnn_pack_bf16")
                parts.append(out)
            # the line pool's key MLP: W1 (d x d) with the value projection
            # (d x d) stacked under it, then W2 (1 x d) zero-padded to 32 rows,
            # then its bias as 32 float32 (the first the real one)
            w1 = np.ascontiguousarray(np.concatenate(
                [np.asarray(weights["line_pool.wk.0.weight"], np.float32),
                 np.asarray(weights["line_pool.wv.weight"], np.float32)]), np.float32)
            w2 = np.zeros((32, self.d), np.float32)
            w2[0] = np.asarray(weights["line_pool.wk.2.weight"], np.float32).reshape(-1)
            b2 = np.zeros(32, np.float32)
            b2[0] = float(np.asarray(weights["line_pool.wk.2.bias"], np.float32).reshape(-1)[0])
            for w in (w1, w2):
                out = np.empty(w.size, np.uint16)
                _lib.check(lib.latec_gnn_pack_bf16(w.ctypes.data, w.shape[0], w.shape[1],
                                                   w.shape[1], out.ctypes.data),
                           "latec_gnn_pack_bf16")
                parts.append(out)
            parts.append(b2.view(np.uint16))
            self.packed = torch.from_numpy(np.concatenate(parts).view(np.int16)).to(self.device)
            m.packed_bf16 = self.packed.data_ptr()
            m.tc_err = self.tc_err.data_ptr()
        elif precision == "fp8":
            parts, scales = [], []
            for name in ("bidir.net.0", "bidir.net.2", "dir.net.0", "dir.net.2", "mix.net.0",
                         "mix.net.2"):
                w = np.ascontiguousarray(weights[name + ".weight"], np.float32)
                n, k = w.shape
                kp = -(-k // 32) * 32
                out = np.empty(n * kp, np.uint8)
                sc = np.empty(n, np.float32)
                _lib.check(lib.latec_gnn_pack_fp8(w.ctypes.data, n, k, kp, out.ctypes.data,
                                                  sc.ctypes.data), "latec_gnn_pack_fp8")
                parts.append(out)
                scales.append(sc)
            self.packed = torch.from_numpy(np.concatenate(parts)).to(self.device)
            self.fp8_scales = torch.from_numpy(np.concatenate(scales)).to(self.device)
            m.packed_fp8 = self.packed.data_ptr()
            m.fp8_scales = self.fp8_scales.data_ptr()
            m.tc_err = self.tc_err.data_ptr()
        self.struct = m
        self._ws = None
        self._lib = lib
        self._ct = ctypes

    def _workspace(self, nbytes):
        torch = _torch()
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.device)
        return self._ws

    def embed(self, E, geom: StageGeom):
        """Per-axis contexts (B, M, K, d) at the stage's queries (GNN.embed)."""
        torch = _torch()
        from . import _lib

        B, N, K, d = E.shape
        ctx = torch.empty((B, geom.M, K, d), dtype=torch.float32, device=self.device)
        ws = self._workspace(self._lib.latec_gnn_workspace_bytes(d, B, geom.M, geom.L, K,
                                                                 geom.m_tile))
        _lib.check(self._lib.latec_gnn_embed(self._ct.byref(self.struct), B, N, E.data_ptr(),
                                             self._ct.byref(geom.struct), ctx.data_ptr(),
                                             ws.data_ptr(), ws.numel(), _lib.stream_ptr()),
                   "latec_gnn_embed")
        return ctx

    def head_of(self, ctx, eb):
        """(mu, log2 b), each (B, M): axis pool + PredHead (GNN.head_of)."""
        torch = _torch()
        from . import _lib

        B, M, K, d = ctx.shape
        mu = torch.empty((B, M), dtype=torch.float32, device=self.device)
        lb = torch.empty((B, M), dtype=torch.float32, device=self.device)
        ws = self._workspace(self._lib.latec_gnn_workspace_bytes(d, B, M, 1, K, 1))
        _lib.check(self._lib.latec_gnn_head(self._ct.byref(self.struct), B, M, K, ctx.data_ptr(),
                                            float(eb), mu.data_ptr(), lb.data_ptr(), ws.data_ptr(),
                                            ws.numel(), _lib.stream_ptr()), "latec_gnn_head")
        return mu, lb

    def finalize(self, ctx, vals, geom: StageGeom, E):
        """Write the revealed points' finalised embeddings into E in place."""
        torch = _torch()
        from . import _lib

        B, M, K, d = ctx.shape
        v = vals.to(device=self.device, dtype=torch.float32).contiguous()
        ws = self._workspace(self._lib.latec_gnn_workspace_bytes(d, B, M, 1, K, 1))
        _lib.check(self._lib.latec_gnn_finalize(self._ct.byref(self.struct), B, E.shape[1], M, K,
                                                geom._t["query"].data_ptr(), ctx.data_ptr(),
                                                v.data_ptr(), E.data_ptr(), ws.data_ptr(),
                                                ws.numel(), _lib.stream_ptr()),
                   "latec_gnn_finalize")
        return E


def stage_forward(model: GNNModel, E, geom_prev, geom_head, finalize_vals, torch=None,
                  finalize_ctx=None, eb=0.01):
    """One codec stage (``latec/gnn_predictor.py:984-1000``): finalise the
    previous stage's revealed points, then predict this stage's queries.
    Returns ``((mu, log_b), E, head_ctx)``."""
    if geom_prev is not None and geom_prev.M:
        ctx = finalize_ctx if finalize_ctx is not None else model.embed(E, geom_prev)
        model.finalize(ctx, finalize_vals, geom_prev, E)
    head_ctx = model.embed(E, geom_head)
    return model.head_of(head_ctx, eb), E, head_ctx


def run_stages(model: GNNModel, x, geoms, eb=0.01):
    """Closed loop over every stage of a (B, *S) field, revealing the true
    values after each stage; returns the per-stage (mu, log_b) and E."""
    torch = _torch()
    xt = torch.as_tensor(x).to(device=model.device, dtype=torch.float32)
    B = xt.shape[0]
    flat = xt.reshape(B, -1)
    E = torch.zeros((B, flat.shape[1], xt.dim() - 1, model.d), dtype=torch.float32,
                    device=model.device)
    out, prev, ctx = [], None, None
    for g in geoms:
        vals = flat[:, prev.query_idx] if prev is not None else None
        (mu, lb), E, ctx = stage_forward(model, E, prev, g, vals, finalize_ctx=ctx, eb=eb)
        out.append((mu, lb))
        prev = g
    return out, E
