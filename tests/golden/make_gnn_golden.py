"""Generate tests/golden/gnn.npz from the reference GNN predictor itself.

Imports the reference package (the checkout's root is the required --ref
argument) with the test-only zstandard shim, loads seeded weights from
``latec_b200.gnn.random_weights`` into ``latec.gnn_predictor.build_model``,
builds the stage geometry with ``build_stage_geoms`` and runs the closed loop
``stage_forward`` over every stage (true values revealed after each stage),
in float32 on the CPU -- the reference's own precision. Stores per case:
per-stage query indices and neighbour steps/validity (pins the geometry), the
per-stage (mu, log2 b), and the first four channels of the final embeddings.

    python tests/golden/make_gnn_golden.py [--ref PATH]
"""

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

CASES = [
    # name, shape, levels, stride, block, max_radius, agg_level, batch, eb, weight seed
    ("g2d", (19, 24), 3, 8, 1, 64, 1, 2, 0.01, 7),
    ("g3d", (9, 10, 8), 2, 4, 1, 16, 1, 1, 0.003, 11),
    ("g2d_agg2", (13, 11), 2, 4, 1, 64, 2, 1, 0.02, 5),
    ("g2d_radius2", (20, 20), 3, 8, 1, 2, 1, 1, 0.01, 3),
]


def field(shape, batch, seed):
    rs = np.random.RandomState(seed)
    grids = np.meshgrid(*[np.linspace(0, 1, n) for n in shape], indexing="ij")
    out = []
    for b in range(batch):
        f = sum(np.sin((2 + b + k) * 3.1 * g + rs.rand() * 6) for k, g in enumerate(grids))
        f = f + 0.05 * rs.randn(*shape)
        out.append((f - f.min()) / (f.max() - f.min()))
    return np.stack(out).astype(np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference LATEC checkout")
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(HERE, "_refshim"))
    sys.path.insert(0, args.ref)
    sys.path.insert(0, ROOT)
    import torch
    from latec.gnn_predictor import build_model, build_stage_geoms, stage_forward

    from latec_b200.gnn import random_weights

    arrays, meta = {}, []
    for name, shape, lv, st, blk, rad, agg, B, eb, wseed in CASES:
        w = random_weights(wseed, 64, agg)
        model = build_model(64, agg).eval()
        model.load_state_dict({k: torch.as_tensor(np.asarray(v)) for k, v in w.items()})
        geoms, _ = build_stage_geoms(shape, lv, st, blk, rad, torch, agg_level=agg)
        x = field(shape, B, wseed)
        flat = torch.from_numpy(x.reshape(B, -1))
        E = torch.zeros(B, flat.shape[1], len(shape), 64)
        prev, ctx = None, None
        for s, g in enumerate(geoms):
            vals = flat[:, prev.idx_np] if prev is not None else None
            with torch.no_grad():
                (mu, lb), E, ctx = stage_forward(model, E, prev, g, vals, torch,
                                                 finalize_ctx=ctx, eb=eb)
            arrays[f"{name}_q{s}"] = g.idx_np.astype(np.int64)
            for k in ("sp", "sn"):
                arrays[f"{name}_{k}{s}"] = getattr(g, k).numpy().astype(np.int32)
            for k in ("vp", "vn"):
                arrays[f"{name}_{k}{s}"] = getattr(g, k).numpy().astype(bool)
            arrays[f"{name}_mu{s}"] = mu.numpy().astype(np.float32)
            arrays[f"{name}_lb{s}"] = lb.numpy().astype(np.float32)
            prev = g
        arrays[f"{name}_x"] = x
        arrays[f"{name}_E"] = E[..., :4].numpy().astype(np.float32)
        meta.append(dict(name=name, shape=list(shape), levels=lv, stride=st, block=blk,
                         max_radius=rad, agg_level=agg, batch=B, eb=eb, seed=wseed,
                         stages=len(geoms)))
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    out = os.path.join(HERE, "gnn.npz")
    np.savez_compressed(out, **arrays)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
