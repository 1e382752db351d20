"""Pin the CPU oracle to golden vectors produced by the reference LATEC code.

The vectors were generated by importing the reference package itself
(tests/golden/make_golden.py); these tests need no GPU and no reference checkout.
"""

import numpy as np
import pytest

from oracle import codec as ocodec
from oracle import interp as ointerp
from oracle import levels as olevels
from oracle import quant as oquant
from oracle import rans_model as orm
from tests.golden_io import codec_case_names, load_npz, schedule_cases, sha


def _field_for(name, z):
    if "x" in z:
        return z["x"]
    from latec_b200 import fields

    if name == "cfg1_512x512":
        x = fields.grf_se((512, 512), 16.0, seed=0)
    elif name == "turb3d_64_rel1e-4":
        x = fields.turbulence_jumps((64, 64, 64), seed=6)
    else:  # pragma: no cover
        raise KeyError(name)
    assert sha(x.astype("<f4")) == bytes(z["x_sha"]).hex()
    return x


@pytest.mark.parametrize("case", schedule_cases(), ids=lambda c: f"{c['shape']}-{c['levels']}-{c['stride']}-{c['block']}")
def test_schedule_matches_reference(case):
    shape, lv, st, blk = tuple(case["shape"]), case["levels"], case["stride"], case["block"]
    assert olevels.stage_counts(shape, lv, st, blk) == case["counts"]
    assert olevels.stage_strides(len(shape), lv, st) == case["strides"]
    assert [float(v) for v in olevels.stage_ebs(shape, lv, st, blk, 1e-3, 0.9)] == case["ebs"]
    if "mask_sha" in case:
        got = [sha(np.flatnonzero(m).astype("<i8")) for m in olevels.stage_masks(shape, lv, st, blk)]
        assert got == case["mask_sha"]


def test_quantizer_matches_reference():
    z = load_npz("quantizer.npz")
    for i, c in enumerate(z["meta"]):
        codes, out = oquant.quantize(z[f"x{i}"], z[f"p{i}"], c["eb"], c["radius"])
        assert np.array_equal(codes, z[f"c{i}"])
        assert np.array_equal(out.view(np.uint32), z[f"o{i}"].view(np.uint32))
        rec = oquant.dequantize(z[f"p{i}"], codes, out, c["eb"], c["radius"])
        assert np.array_equal(rec.view(np.uint32), z[f"r{i}"].view(np.uint32))
    codes, out = oquant.quantize(z["xt"], z["pt"], 0.1)
    assert np.array_equal(codes, z["ct"]) and np.array_equal(out, z["ot"])


def test_predictions_match_reference():
    z = load_npz("predict.npz")
    recon = z["recon2d"]
    shape = recon.shape[1:]
    for order in ("linear", "cubic"):
        for center in (0, 1, 2):
            for em in (0, 1, 2, 3):
                for t, (mask, s, axes) in enumerate(olevels.iter_plan(shape, 3, 8, 1)):
                    key = f"p2d_{order}_{center}_{em}_{t}"
                    if key in z:
                        got = ointerp.predict(recon, s, axes, np.flatnonzero(mask), order, center, em)
                        assert np.array_equal(got, z[key]), key
    recon3 = z["recon3d"]
    for center in (0, 1, 2):
        for em in (0, 3):
            for t, (mask, s, axes) in enumerate(olevels.iter_plan(recon3.shape[1:], 2, 4, 1)):
                key = f"p3d_{center}_{em}_{t}"
                if key in z:
                    got = ointerp.predict(recon3, s, axes, np.flatnonzero(mask), "cubic", center, em)
                    assert np.array_equal(got, z[key]), key


def test_rans_tables_match_reference():
    z = load_npz("rans.npz")
    meta = z["meta"]
    for t in meta["tables"]:
        cdfs = orm.build_cdfs(t["kexp"], t["shape"], owx=t["owx"])
        assert sha(cdfs.astype("<u4")) == t["sha"], t
        key = f"cdf_{t['kexp']}_{t['shape']}_{t['owx']}"
        if key in z:
            assert np.array_equal(cdfs, z[key])
    assert np.array_equal(orm.neg_log2_weights(3, 5, owx=2), z["neglog2_3_5_2"])
    for i, c in enumerate(meta["const_level"]):
        codes = z[f"cl_codes_{i}"]
        kexp = orm.choose_kexp(codes, 1 << 15)
        assert kexp == c["kexp"]
        lvl, shp, owx, bits = orm.choose_const_level(codes, 1 << 15, kexp)
        assert (lvl, shp, owx) == (c["level"], c["shape"], c["owx"]) and bits == c["bits"]
        sp = meta["shape_pick"][i]
        shp2 = orm.choose_shape(codes, z[f"sp_levels_{i}"], 1 << 15, kexp)
        assert shp2 == sp["shape"]
        assert orm.model_bits(codes, z[f"sp_levels_{i}"], 1 << 15, kexp, shp2) == sp["model_bits"]
    assert np.array_equal(orm.scale_to_level(z["scales"], 0.01), z["scale_levels"])
    assert np.array_equal(orm.scale_grid(0.01), z["scale_grid"])
    got = [orm.choose_outlier_weight(a, b) for a, b in
           [(0, 10), (1, 10000), (5, 100), (50, 100), (1, 3), (7, 7000)]]
    assert got == meta["outlier_weight"]


@pytest.mark.parametrize("name", codec_case_names())
def test_codec_stages_match_reference(name):
    z = load_npz(f"codec_{name}.npz")
    m = z["meta"]
    x = _field_for(name, z)
    pk, ck = m["predictor"], m["compress"]
    stream, st = ocodec.compress(
        x, m["eb"], order=m["order"], levels_=ck["levels"], anchor_stride=ck["anchor_stride"],
        anchor_block=ck["anchor_block"], radius=ck.get("radius", 1 << 15),
        eb_ratio=ck.get("eb_ratio"), center=pk.get("center"), end_mode=pk.get("end_mode"),
        mode="compat")
    assert (st["center"], st["end_mode"], st["eb_ratio"]) == (m["center"], m["end_mode"], m["eb_ratio"])
    assert len(st["stages"]) == len(m["stages"])
    for t, (got, want) in enumerate(zip(st["stages"], m["stages"])):
        assert sha(got["codes"].astype("<u4")) == want["codes_sha"], t
        assert sha(np.asarray(got["outliers"], np.float32).astype("<f4")) == want["out_sha"], t
        for k in ("kexp", "level", "shape", "owx"):
            assert got[k] == want[k], (t, k)
        assert got["model_bits"] == want["model_bits"]
        if m["full"]:
            assert np.array_equal(got["codes"], z[f"codes_{t}"].astype(np.uint32))
    assert sha(np.asarray(st["recon"], np.float32).astype("<f4")) == m["recon_sha"]
    back = ocodec.decompress(stream)
    assert np.array_equal(np.asarray(back, np.float32).view(np.uint32),
                          np.asarray(st["recon"], np.float32).view(np.uint32))


@pytest.mark.parametrize("mode", ["native", "compat"])
def test_oracle_roundtrip_modes_and_bound(mode):
    from latec_b200 import fields

    x = fields.turbulence_jumps((24, 20, 18), seed=3)
    eb = 1e-3
    stream, st = ocodec.compress(x, eb, levels_=3, anchor_stride=8, mode=mode)
    back = ocodec.decompress(stream)
    assert np.abs(back.astype(np.float64) - x).max() <= eb
    assert np.array_equal(back, st["recon"])


def test_oracle_float64_bound():
    from latec_b200 import fields

    x = fields.turbulence_jumps((20, 22, 18), seed=4).astype(np.float64) * 1000.0
    eb = 1e-7
    stream, st = ocodec.compress(x, eb, levels_=3, anchor_stride=8, mode="native")
    back = ocodec.decompress(stream)
    assert back.dtype == np.float64
    assert np.abs(back - x).max() <= eb
