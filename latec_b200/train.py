"""Training of the learned predictor with hand-written forward and backward
CUDA kernels (the reference's ``scripts/train_gnn.py``).

A training step runs the stage schedule of synthetic fields with teacher
forcing (``run_stages``, train_gnn.py:373-458): at every stage the revealed
values are the truth plus U(-eb, eb) noise, the GNN predicts the next stage's
points, and the loss is the discretised-Laplace code length in bits per point
(``discretized_laplace_nll``, train_gnn.py:195-232) plus ``mse_weight`` times
the squared prediction error (``prediction_sq_err``). The forward pass keeps
its activations on a tape; the backward pass replays it in reverse stage order
(head, message pass, then the finalisation of the previous stage's points,
whose embedding gradient is complete by then). Every op is a kernel of
``latec_b200/csrc/train_kernels.cu``; the weights, their gradients and the
AdamW moments are flat float32 buffers in the reference state_dict order, so
the optimiser (``torch.optim.AdamW`` semantics, lr warm-up then linear decay
over the last 40 %, train_gnn.py:937-950) and the weight EMA (``ModelEMA``,
train_gnn.py:154-192) are one kernel each. torch only holds device memory and
draws the random numbers.

Precision: ``precision="fp32"`` runs every linear layer's GEMMs in float32;
``precision="bf16"`` is the mixed-precision form (the reference trains the
message pass under optional FP16 autocast with a GradScaler,
train_gnn.py:147-150,938): the GEMMs' operands are rounded to BF16 and
accumulated in float32 on the tcgen05 tensor cores (SIMT tiles with the same
rounding for the 1- and 2-wide layers), while the master weights, gradients,
AdamW moments and every non-GEMM op stay float32. BF16 has float32's exponent
range, so no loss scale is kept; a step whose gradient is not finite is
skipped, as GradScaler skips it.

Deliberate difference from the reference trainer: no chunked two-chunk scenes
(``run_chunked_scene``). The
fields come from ``latec_b200.synthetic``, a restatement of the reference's
generator (advection warp included) whose seeded fields equal the
reference's.
"""

from __future__ import annotations

import math

import numpy as np

from . import _lib
from .gnn import build_stage_geoms, param_shapes, random_weights

__all__ = ["Trainer", "sample_noise", "lr_factor", "train"]


def _torch():
    import torch

    return torch


class _Params:
    """Views of the flat parameter (or gradient) buffer by state_dict name."""

    def __init__(self, flat, d, agg_level):
        self.flat = flat
        off = 0
        self.views = {}
        for name, shp in param_shapes(d, agg_level).items():
            n = int(np.prod(shp)) if shp else 1
            self.views[name] = flat[off:off + n]
            off += n
        self.count = off

    def __getitem__(self, name):
        return self.views[name]

    def ptr(self, name):
        return self.views[name].data_ptr()


def sample_noise(batch, noise_range, rng, device):
    """Per-sample teacher-forcing bound, log-uniform in ``noise_range``
    (train_gnn.py:138-144)."""
    torch = _torch()
    lo, hi = noise_range
    u = torch.from_numpy(rng.uniform(math.log(lo), math.log(hi), batch).astype(np.float32))
    return u.exp().to(device)


def lr_factor(step, steps, warmup):
    """Linear warm-up, flat, then linear decay to 0 over the last 40 %
    (train_gnn.py:942-948)."""
    warm = min(1.0, (step + 1) / warmup) if warmup else 1.0
    decay_start = int(steps * 0.6)
    decay = min(1.0, (steps - step) / max(steps - decay_start, 1))
    return warm * decay


class Trainer:
    """Weights, gradients, AdamW moments and the EMA shadow of one model, with
    the kernel-level forward / backward of a teacher-forced stage schedule."""

    def __init__(self, d=64, agg_level=1, weights=None, seed=0, lr=2e-3, weight_decay=1e-3,
                 ema_decay=0.999, mse_weight=1.0, max_radius=64, device=None, precision="fp32"):
        if precision not in ("fp32", "bf16"):
            raise ValueError("precision must be 'fp32' or 'bf16'")
        torch = _torch()
        self.lib = _lib.load()
        self.precision = precision
        bf = precision == "bf16"
        self._tr_linear = self.lib.latec_tr_linear_bf16 if bf else self.lib.latec_tr_linear
        self._tr_linear_bwd = (self.lib.latec_tr_linear_bwd_bf16 if bf
                               else self.lib.latec_tr_linear_bwd)
        self.skipped_steps = 0
        self.d, self.agg_level = int(d), int(agg_level)
        self.h, self.ds = 2 * self.d, max(1, self.d // 4)
        self.de = self.d + self.ds
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        w = weights if weights is not None else random_weights(seed, self.d, self.agg_level)
        shapes = param_shapes(self.d, self.agg_level)
        flat = np.concatenate([np.asarray(w[k], np.float32).reshape(-1) for k in shapes])
        if flat.size != int(self.lib.latec_gnn_param_count(self.d, self.agg_level)):
            raise ValueError("parameter layout does not match the kernels")
        z = lambda: torch.zeros(flat.size, dtype=torch.float32, device=self.device)  # noqa: E731
        self.p = torch.from_numpy(flat).to(self.device)
        self.g, self.m, self.v = z(), z(), z()
        self.ema = self.p.clone() if ema_decay else None
        self.P, self.G = _Params(self.p, self.d, self.agg_level), _Params(self.g, self.d,
                                                                          self.agg_level)
        self.lr, self.wd, self.ema_decay = float(lr), float(weight_decay), float(ema_decay)
        self.mse_weight = float(mse_weight)
        self.max_radius = int(max_radius)
        self.step_count = 0
        self._geoms = {}

    # -------------------------------------------------------------- helpers
    def _s(self):
        return _lib.stream_ptr()

    def _empty(self, *shape):
        torch = _torch()
        return torch.empty(shape, dtype=torch.float32, device=self.device)

    def _zeros(self, *shape):
        torch = _torch()
        return torch.zeros(shape, dtype=torch.float32, device=self.device)

    def _lin(self, X, rows, fin, name, fout, act):
        """(Y, Z) = act(X W^T + b) with the pre-activation kept when act."""
        Y = self._empty(rows, fout)
        Z = self._empty(rows, fout) if act else None
        _lib.check(self._tr_linear(X.data_ptr(), fin, rows, fin, self.P.ptr(name + ".weight"),
                                   self.P.ptr(name + ".bias"), fout, Y.data_ptr(), fout,
                                   1 if act else 0, Z.data_ptr() if act else None, self._s()),
                   "latec_tr_linear")
        return Y, Z

    def _lin_bwd(self, X, rows, fin, name, fout, dY, Z, dX=None, accum=False):
        _lib.check(self._tr_linear_bwd(
            X.data_ptr(), fin, rows, fin, self.P.ptr(name + ".weight"), fout, dY.data_ptr(), fout,
            Z.data_ptr() if Z is not None else None, 1 if Z is not None else 0,
            dX.data_ptr() if dX is not None else None, fin, 1 if accum else 0,
            self.G.ptr(name + ".weight"), self.G.ptr(name + ".bias"), self._s()),
            "latec_tr_linear_bwd")

    def geoms(self, shape, levels, stride):
        key = (tuple(shape), int(levels), int(stride))
        if key not in self._geoms:
            self._geoms[key] = build_stage_geoms(shape, levels, stride, 1, self.max_radius,
                                                 self.agg_level, device=self.device,
                                                 m_tile=1 << 30)[0]
        return self._geoms[key]

    # -------------------------------------------------------------- forward
    def _embed(self, E, N, B, g):
        """GNN.embed with its tape: per-axis contexts (B * M * K, d)."""
        d, K, L, M = self.d, g.K, g.L, g.M
        t = g._t
        np2 = int(g._two_off[1]) if g.struct.n_tiles else 0
        np1 = int(g._one_off[1]) if g.struct.n_tiles else 0
        r2, r1 = B * np2 * K, B * np1 * K
        rows = r2 + r1
        rec = {"g": g, "np2": np2, "np1": np1, "r2": r2, "r1": r1, "rows": rows}
        MS = self._empty(max(rows, 1), d)
        w2, w1 = 2 * self.de + 2, self.de + 2
        for two, npairs, r, w, name, off in ((1, np2, r2, w2, "bidir", 0), (0, np1, r1, w1, "dir", r2)):
            if not r:
                continue
            X = self._empty(r, w)
            _lib.check(self.lib.latec_tr_rows(E.data_ptr(), N, K, d, self.ds,
                                              self.P.ptr("dir_state.table"), self._ct_geom(g),
                                              (t["two"] if two else t["one"]).data_ptr(), npairs, B,
                                              two, X.data_ptr(), w, self._s()), "latec_tr_rows")
            H, Zh = self._lin(X, r, w, name + ".net.0", self.h, True)
            _lib.check(self._tr_linear(H.data_ptr(), self.h, r, self.h,
                                       self.P.ptr(name + ".net.2.weight"),
                                       self.P.ptr(name + ".net.2.bias"), d, MS[off:].data_ptr(), d,
                                       0, None, self._s()), "latec_tr_linear")
            rec[name] = (X, H, Zh, w, npairs, two)
        S1, Zs = self._lin(MS, rows, d, "line_pool.wk.0", d, True) if rows else (None, None)
        n_out = B * M * K
        ctx = self._empty(n_out, d)
        P = self._empty(n_out, L + 1)
        cand = _torch().empty(n_out * L, dtype=_torch().int32, device=self.device)
        _lib.check(self.lib.latec_tr_line_rows(t["row_of"].data_ptr(), M, L, K, B, np2, np1,
                                               cand.data_ptr(), self._s()), "latec_tr_line_rows")
        if rows:
            KEY, _ = self._lin(S1, rows, d, "line_pool.wk.2", 1, False)
            V, _ = self._lin(MS, rows, d, "line_pool.wv", d, False)
        else:
            KEY, V = self._zeros(1), self._zeros(1, d)
        _lib.check(self.lib.latec_tr_attn(KEY.data_ptr(), V.data_ptr(), d, cand.data_ptr(), L, n_out,
                                          1.0 / math.sqrt(d), self.P.ptr("line_pool.null_k"),
                                          self.P.ptr("line_pool.null_v"), ctx.data_ptr(),
                                          P.data_ptr(), self._s()), "latec_tr_attn")
        rec.update(MS=MS, S1=S1, Zs=Zs, KEY=KEY, V=V, P=P, cand=cand, n_out=n_out)
        return ctx, rec

    def _ct_geom(self, g):
        import ctypes

        return ctypes.byref(g.struct)

    def _head(self, ctx, B, M, K, log_eb):
        d, h = self.d, self.h
        n = B * M
        rows = n * K
        S1, Zs = self._lin(ctx, rows, d, "axis_pool.wk.0", d, True)
        KEY, _ = self._lin(S1, rows, d, "axis_pool.wk.2", 1, False)
        V, _ = self._lin(ctx, rows, d, "axis_pool.wv", d, False)
        pooled = self._empty(n, d)
        P = self._empty(n, K + 1)
        _lib.check(self.lib.latec_tr_attn(KEY.data_ptr(), V.data_ptr(), d, None, K, n,
                                          1.0 / math.sqrt(d), self.P.ptr("axis_pool.null_k"),
                                          self.P.ptr("axis_pool.null_v"), pooled.data_ptr(),
                                          P.data_ptr(), self._s()), "latec_tr_attn")
        X = self._empty(n, d + 1)
        _lib.check(self.lib.latec_tr_head_rows(pooled.data_ptr(), n, M, d, log_eb.data_ptr(),
                                               X.data_ptr(), self._s()), "latec_tr_head_rows")
        H, Zh = self._lin(X, n, d + 1, "head.net.0", h, True)
        O, _ = self._lin(H, n, h, "head.net.2", 2, False)
        mu, lb = self._empty(n), self._empty(n)
        _lib.check(self.lib.latec_tr_head_out(O.data_ptr(), n, M, log_eb.data_ptr(), mu.data_ptr(),
                                              lb.data_ptr(), self._s()), "latec_tr_head_out")
        rec = dict(ctx=ctx, S1=S1, Zs=Zs, KEY=KEY, V=V, P=P, X=X, H=H, Zh=Zh, O=O, mu=mu, n=n,
                   rows=rows, K=K)
        return mu, lb, rec

    def _finalize(self, ctx, vals, g, E, N, B):
        d, h, K, M = self.d, self.h, g.K, g.M
        n = B * M
        rows = n * K
        v = vals.reshape(n, 1).contiguous()
        H1, Z1 = self._lin(v, n, 1, "init.net.0", d, True)
        VE, _ = self._lin(H1, n, d, "init.net.2", d, False)
        X = self._empty(rows, 2 * d)
        _lib.check(self.lib.latec_tr_mix_rows(ctx.data_ptr(), VE.data_ptr(), rows, K, d, X.data_ptr(),
                                              self._s()), "latec_tr_mix_rows")
        H, Zh = self._lin(X, rows, 2 * d, "mix.net.0", h, True)
        Y, _ = self._lin(H, rows, h, "mix.net.2", d, False)
        _lib.check(self.lib.latec_tr_scatter_e(Y.data_ptr(), g._t["query"].data_ptr(), B, M, K, d, N,
                                               E.data_ptr(), 0, self._s()), "latec_tr_scatter_e")
        return dict(g=g, v=v, H1=H1, Z1=Z1, VE=VE, X=X, H=H, Zh=Zh, n=n, rows=rows)

    # -------------------------------------------------------------- backward
    def _embed_bwd(self, rec, dctx, dE, N, B):
        d = self.d
        g = rec["g"]
        rows = rec["rows"]
        dKEY = self._zeros(max(rows, 1))
        dV = self._zeros(max(rows, 1), d)
        _lib.check(self.lib.latec_tr_attn_bwd(rec["V"].data_ptr(), d, rec["cand"].data_ptr(), g.L,
                                              rec["n_out"], 1.0 / math.sqrt(d),
                                              self.P.ptr("line_pool.null_v"), rec["P"].data_ptr(),
                                              dctx.data_ptr(), dKEY.data_ptr(), dV.data_ptr(),
                                              self.G.ptr("line_pool.null_k"),
                                              self.G.ptr("line_pool.null_v"), self._s()),
                   "latec_tr_attn_bwd")
        if not rows:
            return
        MS, S1 = rec["MS"], rec["S1"]
        dMS = self._empty(rows, d)
        self._lin_bwd(MS, rows, d, "line_pool.wv", d, dV, None, dX=dMS)
        dS1 = self._empty(rows, d)
        self._lin_bwd(S1, rows, d, "line_pool.wk.2", 1, dKEY, None, dX=dS1)
        self._lin_bwd(MS, rows, d, "line_pool.wk.0", d, dS1, rec["Zs"], dX=dMS, accum=True)
        for name, off, r in (("bidir", 0, rec["r2"]), ("dir", rec["r2"], rec["r1"])):
            if not r:
                continue
            X, H, Zh, w, npairs, two = rec[name]
            dH = self._empty(r, self.h)
            self._lin_bwd(H, r, self.h, name + ".net.2", d, dMS[off:off + r], None, dX=dH)
            dX = self._empty(r, w)
            self._lin_bwd(X, r, w, name + ".net.0", self.h, dH, Zh, dX=dX)
            _lib.check(self.lib.latec_tr_rows_bwd(dX.data_ptr(), w, N, g.K, d, self.ds,
                                                  self._ct_geom(g),
                                                  (g._t["two"] if two else g._t["one"]).data_ptr(),
                                                  npairs, B, two, dE.data_ptr(),
                                                  self.G.ptr("dir_state.table"), self._s()),
                       "latec_tr_rows_bwd")

    def _head_bwd(self, rec, dmu, dlb, dctx):
        d, h, n, rows, K = self.d, self.h, rec["n"], rec["rows"], rec["K"]
        dO = self._empty(n, 2)
        _lib.check(self.lib.latec_tr_head_out_bwd(rec["O"].data_ptr(), rec["mu"].data_ptr(), n,
                                                  dmu.data_ptr(), dlb.data_ptr(), dO.data_ptr(),
                                                  self._s()), "latec_tr_head_out_bwd")
        dH = self._empty(n, h)
        self._lin_bwd(rec["H"], n, h, "head.net.2", 2, dO, None, dX=dH)
        dX = self._empty(n, d + 1)
        self._lin_bwd(rec["X"], n, d + 1, "head.net.0", h, dH, rec["Zh"], dX=dX)
        dpooled = dX[:, :d].contiguous()
        dKEY, dV = self._zeros(rows), self._zeros(rows, d)
        _lib.check(self.lib.latec_tr_attn_bwd(rec["V"].data_ptr(), d, None, K, n, 1.0 / math.sqrt(d),
                                              self.P.ptr("axis_pool.null_v"), rec["P"].data_ptr(),
                                              dpooled.data_ptr(), dKEY.data_ptr(), dV.data_ptr(),
                                              self.G.ptr("axis_pool.null_k"),
                                              self.G.ptr("axis_pool.null_v"), self._s()),
                   "latec_tr_attn_bwd")
        ctx = rec["ctx"]
        self._lin_bwd(ctx, rows, d, "axis_pool.wv", d, dV, None, dX=dctx, accum=True)
        dS1 = self._empty(rows, d)
        self._lin_bwd(rec["S1"], rows, d, "axis_pool.wk.2", 1, dKEY, None, dX=dS1)
        self._lin_bwd(ctx, rows, d, "axis_pool.wk.0", d, dS1, rec["Zs"], dX=dctx, accum=True)

    def _finalize_bwd(self, rec, dE, dctx, N, B):
        d, h = self.d, self.h
        g, n, rows = rec["g"], rec["n"], rec["rows"]
        dY = self._empty(rows, d)
        _lib.check(self.lib.latec_tr_scatter_e(dY.data_ptr(), g._t["query"].data_ptr(), B, g.M, g.K,
                                               d, N, dE.data_ptr(), 1, self._s()),
                   "latec_tr_scatter_e")
        dH = self._empty(rows, h)
        self._lin_bwd(rec["H"], rows, h, "mix.net.2", d, dY, None, dX=dH)
        dX = self._empty(rows, 2 * d)
        self._lin_bwd(rec["X"], rows, 2 * d, "mix.net.0", h, dH, rec["Zh"], dX=dX)
        dVE = self._zeros(n, d)
        _lib.check(self.lib.latec_tr_mix_rows_bwd(dX.data_ptr(), rows, g.K, d, dctx.data_ptr(),
                                                  dVE.data_ptr(), self._s()),
                   "latec_tr_mix_rows_bwd")
        dH1 = self._empty(n, d)
        self._lin_bwd(rec["H1"], n, d, "init.net.2", d, dVE, None, dX=dH1)
        self._lin_bwd(rec["v"], n, 1, "init.net.0", d, dH1, rec["Z1"], dX=None)

    # -------------------------------------------------------------- a schedule
    def run_stages(self, x, shape, levels, stride, eb, weight=1.0, rng=None, teacher_noise=True):
        """Teacher-forced forward + backward of one batch of fields x (B, N)
        in [0, 1] with per-sample bounds eb (B,); gradients are added to the
        gradient buffer scaled by ``weight / points``. ``teacher_noise=False``
        reveals the exact truth (for gradient checks). Returns (bits per
        point, mse, mae, points)."""
        torch = _torch()
        B, N = x.shape
        K = len(shape)
        geoms = self.geoms(shape, levels, stride)
        npix = B * sum(g.M for g in geoms[1:])
        gen = torch.Generator(device=self.device)
        gen.manual_seed(int(rng.integers(1 << 62)) if rng is not None else 0)
        known = torch.full_like(x, 0.5)

        def reveal(idx):
            if not teacher_noise:
                known[:, idx] = x[:, idx]
                return
            nz = (torch.rand(B, idx.numel(), device=self.device, generator=gen) * 2 - 1) * eb[:, None]
            known[:, idx] = (x[:, idx] + nz).clamp(0.0, 1.0)

        log_eb = torch.log2(eb.clamp_min(1.17549435e-38)).float().contiguous()
        E = self._zeros(B, N, K, self.d)
        acc = torch.zeros(3, dtype=torch.float64, device=self.device)
        scale = float(weight) / max(npix, 1)
        reveal(geoms[0].query_idx)
        ctx0, emb0 = self._embed(E, N, B, geoms[0])
        embs, heads, fins, ctxs, grads = [emb0], [], [], [ctx0], []
        for i in range(1, len(geoms)):
            gp, gh = geoms[i - 1], geoms[i]
            vals = known[:, gp.query_idx].contiguous()
            fins.append(self._finalize(ctxs[i - 1], vals, gp, E, N, B))
            ctx, emb = self._embed(E, N, B, gh)
            embs.append(emb)
            ctxs.append(ctx)
            mu, lb, hr = self._head(ctx, B, gh.M, K, log_eb)
            heads.append(hr)
            tgt = x[:, gh.query_idx].contiguous()
            dmu, dlb = self._empty(B * gh.M), self._empty(B * gh.M)
            _lib.check(self.lib.latec_tr_loss(mu.data_ptr(), lb.data_ptr(), tgt.data_ptr(), B * gh.M,
                                              gh.M, eb.data_ptr(), self.mse_weight, scale,
                                              dmu.data_ptr(), dlb.data_ptr(), acc.data_ptr(),
                                              self._s()), "latec_tr_loss")
            grads.append((dmu, dlb))
            reveal(gh.query_idx)
        # backward: stage i's head and message pass, then the finalisation of
        # stage i - 1's points (their embedding gradient is complete by then)
        dE = self._zeros(B, N, K, self.d)
        dctx = [self._zeros(c.shape[0], self.d) for c in ctxs]
        for i in range(len(geoms) - 1, 0, -1):
            self._head_bwd(heads[i - 1], grads[i - 1][0], grads[i - 1][1], dctx[i])
            self._embed_bwd(embs[i], dctx[i], dE, N, B)
            self._finalize_bwd(fins[i - 1], dE, dctx[i - 1], N, B)
        self._embed_bwd(embs[0], dctx[0], dE, N, B)
        a = acc.cpu().numpy()
        n = max(npix, 1)
        return float(a[0] / n), float(a[1] / n), float(a[2] / n), npix

    # -------------------------------------------------------------- optimiser
    def zero_grad(self):
        self.g.zero_()

    def optimizer_step(self, lr):
        """AdamW (+ EMA) on the float32 master weights. In BF16 mode the
        tensor-core GEMMs' error word is checked first, and a gradient with a
        non-finite entry skips the step (returns False), as GradScaler does."""
        if self.precision == "bf16":
            _lib.check(self.lib.latec_tr_gemm_status(self._s()), "latec_tr_gemm_status")
            if not bool(_torch().isfinite(self.g).all()):
                self.skipped_steps += 1
                return False
        self.step_count += 1
        _lib.check(self.lib.latec_tr_adamw(self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(),
                                           self.v.data_ptr(), self.p.numel(), float(lr), 0.9,
                                           0.999, 1e-8, self.wd, self.step_count, self._s()),
                   "latec_tr_adamw")
        if self.ema is not None:
            s = self.step_count - 1
            decay = min(self.ema_decay, (1.0 + s) / (10.0 + s))
            _lib.check(self.lib.latec_tr_ema(self.ema.data_ptr(), self.p.data_ptr(), self.p.numel(),
                                             float(decay), self._s()), "latec_tr_ema")
        return True

    def weights(self, ema=True):
        """The (EMA) weights as a state_dict of float32 arrays."""
        src = self.ema if (ema and self.ema is not None) else self.p
        flat = src.detach().cpu().numpy()
        out, off = {}, 0
        for name, shp in param_shapes(self.d, self.agg_level).items():
            n = int(np.prod(shp)) if shp else 1
            out[name] = flat[off:off + n].reshape(shp).copy()
            off += n
        return out

    def save(self, path, ema=True):
        """A v7 checkpoint that ``GNNCodec(checkpoint_path=...)`` loads."""
        torch = _torch()
        from .gnn import CKPT_VERSION

        sd = {k: torch.from_numpy(np.asarray(v, np.float32)) for k, v in self.weights(ema).items()}
        torch.save({"version": CKPT_VERSION, "d": self.d, "agg_level": self.agg_level,
                    "state_dict": sd}, path)


def train(steps=3000, *, d=64, agg_level=1, shape4=(16, 16, 16, 16), batch4=4,
          shape2=(128, 128), batch2=16, stride4=8, shape3=(40, 40, 40), batch3=0, stride3=8,
          noise_range=(1e-4, 1e-2), lr=2e-3, warmup=100,
          ema_decay=0.999, mse_weight=1.0, seed=0, device=None, log_every=50, out=None,
          trainer=None, callback=None, synthetic=None, precision="fp32"):
    """Train on mixed 4-D / 2-D synthetic batches (train_h100.sh: 16^4 x 4
    plus 128^2 x 16 per step); returns the Trainer. ``batch3`` > 0 adds 3-D
    fields of ``shape3`` (the 4-D correlation knob, ``stride3``) to every step,
    a mix the reference's script does not train on. ``synthetic`` overrides
    the generator's distribution knobs (``latec_b200.synthetic.DEFAULTS``, the
    reference's synthetic_dist.yaml)."""
    from .synthetic import DEFAULTS, sample_synthetic_batch

    knobs = dict(DEFAULTS, **(synthetic or {}))
    gen = {k: knobs[k] for k in ("turbulence_frac", "max_discontinuities", "discontinuity_frac")}
    corr = {"synthetic": knobs["correlation_4d"], "field2d": knobs["correlation_2d"],
            "field3d": knobs["correlation_4d"]}

    tr = trainer or Trainer(d=d, agg_level=agg_level, seed=seed, lr=lr, ema_decay=ema_decay,
                            mse_weight=mse_weight, device=device, precision=precision)
    rng = np.random.default_rng(seed)
    strides2 = (8, 16, 32)
    hist = []
    for step in range(steps):
        tr.zero_grad()
        logs = {}
        legs = [("synthetic", shape4, batch4, stride4),
                ("field2d", shape2, batch2, int(rng.choice(strides2)))]
        if batch3:
            legs.append(("field3d", shape3, batch3, stride3))
        npts = {k: (math.prod(shp) * b if b else 0) for k, shp, b, _ in legs}
        for kind, shp, bsz, stride in legs:
            if not bsz:
                continue
            x = sample_synthetic_batch(bsz, shp, corr[kind], rng, device=tr.device, **gen)
            eb = sample_noise(bsz, noise_range, rng, tr.device)
            levels = stride.bit_length() - 1
            w = npts[kind] / max(sum(npts.values()), 1)
            bits, mse, mae, _ = tr.run_stages(x, shp, levels, stride, eb, weight=w, rng=rng)
            logs[kind] = (bits, mse, mae)
        tr.optimizer_step(tr.lr * lr_factor(step, steps, warmup))
        hist.append(logs)
        if callback is not None:
            callback(step, logs)
        if log_every and (step % log_every == 0 or step == steps - 1):
            parts = " ".join(f"{k}: {v[0]:.3f} bpp mse {v[1]:.2e}" for k, v in logs.items())
            print(f"step {step}: {parts}", flush=True)
    if out:
        tr.save(out)
    return tr, hist


def main(argv=None):
    import argparse

    ap = argparse.ArgumentParser(description="train the axial GNN predictor on synthetic fields")
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--d", type=int, default=64)
    ap.add_argument("--agg-level", type=int, default=1)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--ema-decay", type=float, default=0.999)
    ap.add_argument("--mse-weight", type=float, default=1.0)
    ap.add_argument("--batch4", type=int, default=4)
    ap.add_argument("--batch2", type=int, default=16)
    ap.add_argument("--batch3", type=int, default=0)
    ap.add_argument("--shape3", type=int, nargs=3, default=(40, 40, 40))
    ap.add_argument("--noise-range", type=float, nargs=2, default=(1e-4, 1e-2))
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default="gnn_trained.pt")
    ap.add_argument("--precision", choices=("fp32", "bf16"), default="fp32",
                    help="GEMM operands of the linear layers (bf16: tensor cores, float32 "
                         "accumulation and master weights)")
    # the generator's knobs (the reference trainer's --synthetic-* flags)
    ap.add_argument("--synthetic-turbulence-frac", type=float, default=None)
    ap.add_argument("--synthetic-discontinuities", type=int, default=None)
    ap.add_argument("--synthetic-discontinuity-frac", type=float, default=None)
    ap.add_argument("--synthetic-correlation", type=float, nargs=2, default=None)
    ap.add_argument("--synthetic-2d-correlation", type=float, nargs=2, default=None)
    a = ap.parse_args(argv)
    given = {"turbulence_frac": a.synthetic_turbulence_frac,
             "max_discontinuities": a.synthetic_discontinuities,
             "discontinuity_frac": a.synthetic_discontinuity_frac,
             "correlation_4d": a.synthetic_correlation,
             "correlation_2d": a.synthetic_2d_correlation}
    train(a.steps, d=a.d, agg_level=a.agg_level, lr=a.lr, warmup=a.warmup, ema_decay=a.ema_decay,
          mse_weight=a.mse_weight, batch4=a.batch4, batch2=a.batch2, batch3=a.batch3,
          shape3=tuple(a.shape3),
          noise_range=tuple(a.noise_range), seed=a.seed, out=a.out, precision=a.precision,
          synthetic={k: v for k, v in given.items() if v is not None})


if __name__ == "__main__":
    main()
