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
