"""Generate tests/golden/gnn_codec.npz from the reference learned codec itself.

Imports the reference package (root given by the required --ref argument)
with the test-only zstandard shim and runs ``latec.GNNCodec.compress`` on the
CPU in float32 (``fp16=False``, gate on) with the checkpoint this repository
ships (``latec_b200/checkpoints/gnn_d64_agg1_synthetic.pt``, written in the
reference's v7 checkpoint format, so the reference loads it as its own).
The rANS packing (``pack_stage``; its coder, the ``constriction`` crate, is
not installed) is replaced by a recorder, and the per-stage device steps of
``_compress_chunked`` (latec/gnn_codec.py:1048-1336) are wrapped to record,
per stage: the model's mu and scale, the gate's choice (kind, direction, T,
shift), the gated prediction and scale, the codes, the outliers and the scale
levels; plus the anchor stage's codes and the final normalised
reconstruction. Single-chunk cases in 2-D, 3-D and 4-D, two of them with
``gate_fine`` (one gate chosen at the first finest sub-stage and reused by the
others: no choice is recorded for those).

    python tests/golden/make_gnn_codec_golden.py --ref PATH
"""

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CKPT = os.path.join(ROOT, "latec_b200", "checkpoints", "gnn_d64_agg1_synthetic.pt")

CASES = [
    # name, shape, levels, absolute eb, field, gate_fine
    ("c2d", (48, 40), 3, 1e-3, "grf", False),
    ("c3d", (16, 16, 20), 3, 1e-3, "turb", False),
    ("c4d", (8, 8, 10, 8), 2, 1e-3, "mixed", False),
    ("c2d_l4", (40, 36), 4, 3e-4, "mixed2d", False),
    # one gate descriptor shared by the finest level's sub-stages
    ("c3d_fine", (16, 20, 16), 3, 1e-3, "turb", True),
    ("c2d_fine", (40, 48), 3, 5e-4, "mixed2d", True),
]


def make_field(kind, shape, seed):
    sys.path.insert(0, ROOT)
    from latec_b200 import fields

    if kind == "grf":
        return fields.grf_se(shape, 6.0, seed=seed)
    if kind == "turb":
        return fields.turbulence_jumps(shape, seed=seed)
    if kind == "mixed2d":
        a = fields.grf_aniso(shape, (3.0, 7.0), seed=seed)
        b = fields.turbulence_jumps(shape, seed=seed + 1)
        return (0.5 * a + 0.5 * b).astype(np.float32)
    return fields.mixed_4d(shape, seed=seed)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference LATEC checkout")
    ap.add_argument("--out", default=os.path.join(HERE, "gnn_codec.npz"))
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(HERE, "_refshim"))
    sys.path.insert(0, args.ref)
    import torch

    torch.set_num_threads(8)
    import latec.gnn_codec as gc
    import latec.gnn_predictor as gp

    rec = {"stages": [], "anchor": None, "recon": None}
    cur = {}

    orig_pred = gp.ChunkedGNNPredictor.predict_wave_stage

    def pred_rec(self, s, recon_t, eb):
        pred, scale = orig_pred(self, s, recon_t, eb)
        cur.clear()
        cur.update(s=s, eb=float(eb), mu=pred[0].reshape(-1).clone(),
                   scale=scale[0].reshape(-1).clone())
        return pred, scale

    orig_select = gc._gate_select_t

    def select_rec(torch_, r_g, r_is, b, eb, radius=1 << 15):
        out = orig_select(torch_, r_g, r_is, b, eb, radius)
        cur["gate"] = [int(v) for v in out]
        return out

    orig_apply = gc._gate_apply_t

    def apply_rec(torch_, pred_bi, scale_bi, ip, eb, gate_t, gate_sh, gate_dir):
        p, sc = orig_apply(torch_, pred_bi, scale_bi, ip, eb, gate_t, gate_sh, gate_dir)
        cur["mu_g"] = p.reshape(-1).clone()
        cur["scale_g"] = sc.reshape(-1).clone()
        return p, sc

    orig_quant = gc._quantize_t

    def quant_rec(torch_, x, pred, eb, radius, round_output):
        codes, recon, outl = orig_quant(torch_, x, pred, eb, radius, round_output)
        cur["x"] = x.reshape(-1).clone()
        cur["codes"] = codes.reshape(-1).clone()
        cur["outliers"] = outl.reshape(-1).clone()
        return codes, recon, outl

    orig_lv = gc._scale_to_level_t

    def lv_rec(torch_, scale, eb):
        lv = orig_lv(torch_, scale, eb)
        cur["levels"] = lv.reshape(-1).clone()
        rec["stages"].append(dict(cur))
        return lv

    orig_anchor = gc._code_anchor_stage

    def anchor_rec(values, axes, eb0, radius, round_output, norm):
        packed, recon = orig_anchor(values, axes, eb0, radius, round_output, norm)
        rec["anchor"] = np.asarray(recon).reshape(-1).copy()
        return packed, recon

    orig_finish = gp.ChunkedGNNPredictor.finish_wave

    def finish_rec(self, recon_t):
        rec["recon"] = recon_t.detach().cpu().numpy().reshape(-1).copy()
        return orig_finish(self, recon_t)

    gp.ChunkedGNNPredictor.predict_wave_stage = pred_rec
    gp.ChunkedGNNPredictor.finish_wave = finish_rec
    gc._gate_select_t = select_rec
    gc._gate_apply_t = apply_rec
    gc._quantize_t = quant_rec
    gc._scale_to_level_t = lv_rec
    gc._code_anchor_stage = anchor_rec
    import latec.bitstream as bs

    def fake_pack(codes, outliers, **kw):
        return b""

    gc.pack_stage = fake_pack
    bs.pack_stage = fake_pack

    from latec.gnn_codec import GNNCodec

    codec = GNNCodec(CKPT, device="cpu")
    arrays, meta = {}, []
    for ci, (name, shape, levels, eb_abs, kind, fine) in enumerate(CASES):
        x = np.ascontiguousarray(make_field(kind, shape, 100 + ci), np.float32)
        span = float(np.float32(x.max())) - float(np.float32(x.min()))
        rel = eb_abs / span
        rec["stages"], rec["anchor"], rec["recon"] = [], None, None
        codec.compress(x, rel, levels=levels, fp16=False, gate=True, gate_fine=fine,
                       compile=False)
        st = rec["stages"]
        arrays[f"{name}/x"] = x
        arrays[f"{name}/anchor_recon"] = rec["anchor"].astype(np.float32)
        arrays[f"{name}/recon"] = rec["recon"].astype(np.float32)
        gates = []
        for k, d in enumerate(st):
            for key in ("mu", "scale", "outliers", "mu_g", "scale_g"):
                arrays[f"{name}/{k}/{key}"] = d[key].numpy().astype(np.float32)
            arrays[f"{name}/{k}/codes"] = d["codes"].numpy().astype(np.int32)
            arrays[f"{name}/{k}/levels"] = d["levels"].numpy().astype(np.uint8)
            gates.append(d.get("gate"))
        meta.append({"name": name, "shape": list(shape), "levels": levels, "rel_eb": rel,
                     "eb_abs": eb_abs, "gate_fine": fine, "stages": [d["s"] for d in st],
                     "ebs": [d["eb"] for d in st], "gates": gates})
        print(name, shape, "stages", len(st), "gates", gates, flush=True)
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    np.savez_compressed(args.out, **arrays)
    print("wrote", args.out, os.path.getsize(args.out), "bytes")


if __name__ == "__main__":
    main()
