"""Generate the golden vectors that pin the oracle to the reference LATEC code.

Run in a container that has the reference checkout (read-only is fine):

    python tests/golden/make_golden.py --reference <reference checkout>

It imports the reference package itself (``latec``) with two test-only
stand-ins on ``sys.path``: ``_refshim/zstandard.py`` (ctypes over the system
libzstd) because python-zstandard is not installed, and a recorder in place of
``latec.codec.pack_stage`` because the rANS back end (``constriction``) is not
installed either. The recorder captures, per stage, exactly what the reference
hands to its entropy stage -- codes and outliers in scan order -- plus the
stage-constant model choice the reference computes from them
(``choose_kexp`` / ``choose_const_level``, pure NumPy), then returns an empty
payload. ``stats["recon"]`` is the reference's own closed-loop reconstruction.

Nothing here is imported by the package, the tests at run time, or the bench:
the tests read only the ``.npz`` files this script writes.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _import_reference(ref_root: str):
    sys.path.insert(0, os.path.join(HERE, "_refshim"))
    sys.path.insert(0, ref_root)
    import latec.codec as codec  # noqa: F401  (reference package)
    import latec.levels as levels
    import latec.predictor as predictor
    import latec.quantizer as quantizer
    import latec.rans as rans

    return codec, levels, predictor, quantizer, rans


def _record_compress(codec, rans, x, eb, pred_obj, **kw):
    """Run the reference ``compress`` with the entropy stage recorded."""
    rec = []
    real = codec.pack_stage

    def fake_pack_stage(codes, outliers, *, rans_levels=None, rans_tables=None,
                        radius=1 << 15, zstd_level=9):
        codes = np.asarray(codes, np.uint32).copy()
        outliers = np.asarray(outliers, np.float32).copy()
        tables = rans.const_tables(radius)
        kexp = rans.choose_kexp(codes, tables.radius)
        level, shape, owx, bits = rans.choose_const_level(codes, tables, kexp)
        rec.append(dict(codes=codes, outliers=outliers, kexp=int(kexp),
                        level=int(level), shape=int(shape), owx=int(owx),
                        model_bits=float(bits)))
        return b""

    codec.pack_stage = fake_pack_stage
    try:
        _stream, stats = codec.compress(x, eb, pred_obj, **kw)
    finally:
        codec.pack_stage = real
    return rec, stats


# (name, field builder, eb, predictor kwargs, compress kwargs, keep full arrays)
def _cases():
    from latec_b200 import fields

    rs = np.random.RandomState(7)
    nan_field = fields.grf_se((40, 36), corr_len=5.0, seed=3)
    nan_field[3, 5] = np.nan
    nan_field[20, 20] = np.inf
    nan_field[33, 1] = -np.inf
    big_range = (rs.randn(48, 40) * 1e4).astype(np.float32)
    return [
        ("cfg1_512x512", lambda: fields.grf_se((512, 512), 16.0, seed=0), 1e-3,
         dict(order="cubic", levels=4, anchor_stride=16, anchor_block=1),
         dict(levels=4, anchor_stride=16, anchor_block=1), False),
        ("grf2d_128", lambda: fields.grf_se((128, 128), 8.0, seed=1), 1e-3,
         dict(order="cubic", levels=4, anchor_stride=16, anchor_block=1),
         dict(levels=4, anchor_stride=16, anchor_block=1), True),
        ("odd2d_linear_flat", lambda: fields.grf_se((37, 53), 4.0, seed=2), 2e-3,
         dict(order="linear", levels=3, anchor_stride=8, anchor_block=1, center=0, end_mode=0),
         dict(levels=3, anchor_stride=8, anchor_block=1, eb_ratio=1.0), True),
        *[
            (f"odd3d_c{c}_e{e}", (lambda: fields.turbulence_jumps((33, 20, 17), seed=4)), 1e-2,
             dict(order="cubic", levels=3, anchor_stride=8, anchor_block=1, center=c, end_mode=e),
             dict(levels=3, anchor_stride=8, anchor_block=1), True)
            for c in (0, 1, 2) for e in (0, 1, 2, 3)
        ],
        ("odd3d_linear_extrap", lambda: fields.turbulence_jumps((21, 18, 25), seed=5), 5e-3,
         dict(order="linear", levels=3, anchor_stride=8, anchor_block=1, center=0, end_mode=3),
         dict(levels=3, anchor_stride=8, anchor_block=1, eb_ratio=0.7), True),
        ("turb3d_64_rel1e-4", lambda: fields.turbulence_jumps((64, 64, 64), seed=6), None,
         dict(order="cubic", levels=6, anchor_stride=64, anchor_block=1),
         dict(levels=6, anchor_stride=64, anchor_block=1), False),
        ("grf4d_default_center", lambda: fields.grf_se((9, 10, 11, 12), 3.0, seed=8), 1e-2,
         dict(order="cubic", levels=2, anchor_stride=4, anchor_block=1),
         dict(levels=2, anchor_stride=4, anchor_block=1), True),
        ("grf4d_center0_extrap", lambda: fields.grf_se((8, 7, 9, 10), 3.0, seed=9), 1e-2,
         dict(order="cubic", levels=3, anchor_stride=8, anchor_block=1, center=0, end_mode=3),
         dict(levels=3, anchor_stride=8, anchor_block=1), True),
        ("line_1x1000", lambda: fields.grf_se((1, 1000), 20.0, seed=10), 1e-3,
         dict(order="cubic", levels=5, anchor_stride=32, anchor_block=1),
         dict(levels=5, anchor_stride=32, anchor_block=1), True),
        ("thin_17x1x9", lambda: fields.grf_se((17, 1, 9), 3.0, seed=11), 1e-2,
         dict(order="cubic", levels=3, anchor_stride=8, anchor_block=1, center=0, end_mode=3),
         dict(levels=3, anchor_stride=8, anchor_block=1), True),
        ("tiny_2x2", lambda: fields.grf_se((2, 2), 1.0, seed=12), 1e-2,
         dict(order="cubic", levels=4, anchor_stride=16, anchor_block=1),
         dict(levels=4, anchor_stride=16, anchor_block=1), True),
        ("extra_levels", lambda: fields.grf_se((30, 26), 4.0, seed=13), 1e-3,
         dict(order="cubic", levels=5, anchor_stride=8, anchor_block=1),
         dict(levels=5, anchor_stride=8, anchor_block=1), True),
        ("nan_inf_2d", lambda: nan_field, 1e-2,
         dict(order="cubic", levels=3, anchor_stride=8, anchor_block=1, end_mode=3),
         dict(levels=3, anchor_stride=8, anchor_block=1), True),
        ("small_radius", lambda: big_range, 1.0,
         dict(order="cubic", levels=3, anchor_stride=8, anchor_block=1),
         dict(levels=3, anchor_stride=8, anchor_block=1, radius=64), True),
        ("image_3ch", lambda: (np.random.RandomState(14).rand(24, 31, 3) * 100).astype(np.float32),
         0.5, dict(order="cubic", levels=3, anchor_stride=8, anchor_block=1),
         dict(levels=3, anchor_stride=8, anchor_block=1), True),
        # blocked anchors: anchor_block^ndim blocks on the anchor lattice, the
        # finer stages skip them (InterpPredictor's own default block is 4)
        ("block4_2d", lambda: fields.grf_se((45, 38), 5.0, seed=15), 1e-3,
         dict(order="cubic", levels=4, anchor_stride=8, anchor_block=4),
         dict(levels=4, anchor_stride=8, anchor_block=4), True),
        ("block4_3d", lambda: fields.turbulence_jumps((21, 30, 19), seed=16), 5e-3,
         dict(order="cubic", levels=3, anchor_stride=8, anchor_block=4, center=0, end_mode=3),
         dict(levels=3, anchor_stride=8, anchor_block=4), True),
        ("block2_4d", lambda: fields.grf_se((9, 8, 10, 7), 3.0, seed=17), 1e-2,
         dict(order="cubic", levels=2, anchor_stride=4, anchor_block=2),
         dict(levels=2, anchor_stride=4, anchor_block=2), True),
        ("block3_2d_linear", lambda: fields.grf_se((33, 29), 4.0, seed=18), 2e-3,
         dict(order="linear", levels=3, anchor_stride=8, anchor_block=3, center=0, end_mode=1),
         dict(levels=3, anchor_stride=8, anchor_block=3), True),
    ]


def make_codec_cases(codec, rans, predictor_mod, out_dir):
    index = {}
    for name, build, eb, pkw, ckw, full in _cases():
        x = build()
        if eb is None:  # relative bound, as the reference CLI computes it
            eb = 1e-4 * (float(np.max(x.astype(np.float64))) - float(np.min(x.astype(np.float64))))
        pkw = dict(pkw)
        order = pkw.pop("order")
        pred = predictor_mod.InterpPredictor(order, **pkw)
        rec, stats = _record_compress(codec, rans, x, eb, pred, **ckw)
        meta = dict(
            eb=float(eb), order=order, predictor=pkw, compress=ckw,
            center=int(stats["interp_center"]), end_mode=int(stats["interp_end_mode"]),
            eb_ratio=float(stats["eb_ratio"]), shape=list(x.shape),
            stage_codes=[int(v) for v in stats["stage_codes"]],
            stage_outliers=[int(v) for v in stats["stage_outliers"]],
            stages=[dict(kexp=r["kexp"], level=r["level"], shape=r["shape"], owx=r["owx"],
                         model_bits=r["model_bits"], n=int(len(r["codes"])),
                         n_out=int(len(r["outliers"])),
                         codes_sha=_sha(r["codes"].astype("<u4")),
                         out_sha=_sha(r["outliers"].astype("<f4")))
                    for r in rec],
            recon_sha=_sha(np.asarray(stats["recon"], np.float32).astype("<f4")),
            full=bool(full),
        )
        arrays = {}
        if full:
            arrays["x"] = x
            arrays["recon"] = np.asarray(stats["recon"], np.float32)
            for t, r in enumerate(rec):
                arrays[f"codes_{t}"] = r["codes"].astype(np.uint16 if r["codes"].max(initial=0) < 65536 else np.uint32)
                arrays[f"out_{t}"] = r["outliers"]
        else:
            arrays["x_sha"] = np.frombuffer(bytes.fromhex(_sha(x.astype("<f4"))), np.uint8)
        np.savez_compressed(os.path.join(out_dir, f"codec_{name}.npz"), **arrays,
                            meta=np.frombuffer(json.dumps(meta).encode(), np.uint8))
        index[name] = meta["recon_sha"]
        print(f"{name}: {len(rec)} stages, {sum(meta['stage_outliers'])} outliers")
    return index


def make_predict_cases(levels_mod, predictor_mod, out_dir):
    """Multi-channel per-stage predictions on random recon (the reference's own
    whole-grid parity test pattern), for every order/center/end mode."""
    arrays = {}
    shape, lv, stride = (38, 45), 3, 8
    recon = np.random.RandomState(0).rand(2, *shape).astype(np.float32) * 50
    arrays["recon2d"] = recon
    for order in ("linear", "cubic"):
        for center in (0, 1, 2):
            for em in (0, 1, 2, 3):
                p = predictor_mod.InterpPredictor(order, lv, stride, 1, center=center, end_mode=em)
                known = np.zeros(shape, bool)
                for t, (mask, s, axes) in enumerate(levels_mod.stage_plan(shape, lv, stride, 1)):
                    if axes and mask.any():
                        arrays[f"p2d_{order}_{center}_{em}_{t}"] = p.predict(recon, known, mask)
                    known |= mask
    shape3 = (16, 13, 11)
    recon3 = np.random.RandomState(1).rand(1, *shape3).astype(np.float32) * 10
    arrays["recon3d"] = recon3
    for center in (0, 1, 2):
        for em in (0, 3):
            p = predictor_mod.InterpPredictor("cubic", 2, 4, 1, center=center, end_mode=em)
            known = np.zeros(shape3, bool)
            for t, (mask, s, axes) in enumerate(levels_mod.stage_plan(shape3, 2, 4, 1)):
                if axes and mask.any():
                    arrays[f"p3d_{center}_{em}_{t}"] = p.predict(recon3, known, mask)
                known |= mask
    np.savez_compressed(os.path.join(out_dir, "predict.npz"), **arrays)


def make_schedule_cases(levels_mod, out_dir):
    schedules = [
        ((24,), 3, 8, 1), ((64, 64), 3, 8, 1), ((64, 64), 3, 8, 4), ((33, 65), 4, 16, 2),
        ((19, 23, 17), 3, 8, 1), ((16, 16, 16, 16), 4, 16, 1),
        ((17, 16, 16, 16, 16), 4, 16, 1), ((64, 64), 5, 16, 1), ((1, 7), 3, 8, 1),
        ((5, 1, 7), 2, 4, 1), ((512, 512), 4, 16, 1), ((512, 512, 512), 6, 64, 1),
        ((128, 128, 64, 64), 4, 16, 1), ((33, 33, 33, 33), 4, 16, 1),
    ]
    out = []
    for shape, lv, stride, block in schedules:
        entry = dict(shape=list(shape), levels=lv, stride=stride, block=block,
                     counts=levels_mod.stage_counts(shape, lv, stride, block),
                     strides=levels_mod.stage_strides(len(shape), lv, stride),
                     ebs=[float(v) for v in levels_mod.stage_ebs(shape, lv, stride, block, 1e-3, 0.9)])
        if int(np.prod(shape)) <= 1 << 17:
            entry["mask_sha"] = [
                _sha(np.flatnonzero(m).astype("<i8"))
                for m in levels_mod.stage_masks(shape, lv, stride, block)
            ]
        if block == 1:
            entry["layouts"] = [
                [dict(parity=list(c.parity), starts=list(c.starts), step=int(c.step),
                      sizes=list(c.sizes), strides=list(c.strides), offset=int(c.offset))
                 for c in st.classes]
                for st in levels_mod.stage_layouts(shape, lv, stride)
            ]
        out.append(entry)
    with open(os.path.join(out_dir, "schedule.json"), "w") as f:
        json.dump(out, f)


def make_rans_cases(rans, out_dir):
    arrays = {}
    meta = {"tables": [], "const_level": [], "shape_pick": [], "scale": None}
    for kexp in (1, 2, 3, 5, 8, 11, 14):
        for shape in (0, 3, 12, 20):
            if shape not in rans._shape_ids(kexp):
                continue
            for owx in (0, 4, 7):
                cdfs = rans._build_cdfs_cached(kexp, shape, 64, 24, owx)
                key = f"cdf_{kexp}_{shape}_{owx}"
                meta["tables"].append(dict(kexp=kexp, shape=shape, owx=owx, sha=_sha(cdfs.astype("<u4"))))
                if kexp <= 5:
                    arrays[key] = cdfs
    nl = rans._neg_log2_weights(3, 5, 64, 24, 2)
    arrays["neglog2_3_5_2"] = nl
    rs = np.random.RandomState(3)
    for i, (kexp_peak, n, p_out) in enumerate([(3, 5000, 0.0), (6, 20000, 0.01), (1, 300, 0.2),
                                               (10, 7000, 0.001), (14, 3000, 0.0)]):
        q = np.clip(np.round(rs.laplace(0, (1 << kexp_peak) / 6.0, n)), -(1 << kexp_peak) + 1,
                    (1 << kexp_peak) - 1).astype(np.int64)
        codes = (q + (1 << 15)).astype(np.uint32)
        codes[rs.rand(n) < p_out] = 0
        tables = rans.const_tables(1 << 15)
        kexp = rans.choose_kexp(codes, 1 << 15)
        lvl, shp, owx, bits = rans.choose_const_level(codes, tables, kexp)
        arrays[f"cl_codes_{i}"] = codes
        meta["const_level"].append(dict(kexp=int(kexp), level=int(lvl), shape=int(shp),
                                        owx=int(owx), bits=float(bits)))
        levels64 = rs.randint(0, 64, n).astype(np.uint8)
        tables_e = rans.build_laplace_tables(0.01, 1 << 15)
        shp2 = rans.choose_shape(codes, levels64, tables_e, kexp)
        mb = rans.model_bits(codes, levels64, tables_e, kexp=kexp, shape=shp2)
        arrays[f"sp_levels_{i}"] = levels64
        meta["shape_pick"].append(dict(kexp=int(kexp), shape=int(shp2), model_bits=float(mb)))
    scales = np.exp(rs.uniform(np.log(1e-6), np.log(10.0), 4000)).astype(np.float32)
    arrays["scales"] = scales
    arrays["scale_levels"] = rans.scale_to_level(scales, 0.01)
    arrays["scale_grid"] = rans.build_laplace_tables(0.01, 1 << 15).scale_grid
    meta["outlier_weight"] = [rans.choose_outlier_weight(a, b) for a, b in
                              [(0, 10), (1, 10000), (5, 100), (50, 100), (1, 3), (7, 7000)]]
    np.savez_compressed(os.path.join(out_dir, "rans.npz"), **arrays,
                        meta=np.frombuffer(json.dumps(meta).encode(), np.uint8))


def make_quantizer_cases(quantizer, out_dir):
    rs = np.random.RandomState(42)
    arrays = {}
    cases = []
    for i, (scale, eb, radius) in enumerate([(1.0, 0.01, 1 << 15), (255.0, 2.0, 1 << 15),
                                             (1e6, 1e-3, 1 << 15), (1e-3, 1e-7, 1 << 15),
                                             (10.0, 0.01, 16)]):
        x = (rs.randn(5000) * scale).astype(np.float32)
        pred = x + (rs.randn(5000) * eb * 10).astype(np.float32)
        x[::997] = np.float32(1e7)
        codes, outliers = quantizer.quantize(x, pred, eb, radius)
        recon = quantizer.dequantize(pred, codes, outliers, eb, radius)
        arrays.update({f"x{i}": x, f"p{i}": pred, f"c{i}": codes, f"o{i}": outliers, f"r{i}": recon})
        cases.append(dict(eb=eb, radius=radius))
    # tie edges
    pred = np.zeros(9, np.float32)
    x = (np.arange(-4, 5) * 2 + 1).astype(np.float32) * np.float32(0.1)
    codes, outliers = quantizer.quantize(x, pred, 0.1)
    arrays.update({"xt": x, "pt": pred, "ct": codes, "ot": outliers})
    np.savez_compressed(os.path.join(out_dir, "quantizer.npz"), **arrays,
                        meta=np.frombuffer(json.dumps(cases).encode(), np.uint8))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference LATEC checkout")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    codec, levels_mod, predictor_mod, quantizer, rans = _import_reference(args.reference)
    make_schedule_cases(levels_mod, args.out)
    make_quantizer_cases(quantizer, args.out)
    make_rans_cases(rans, args.out)
    make_predict_cases(levels_mod, predictor_mod, args.out)
    make_codec_cases(codec, rans, predictor_mod, args.out)


if __name__ == "__main__":
    main()
