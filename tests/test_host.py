"""Host-side logic and the C ABI library, without a GPU."""

import ctypes
import os
import re

import numpy as np
import pytest

from oracle import ans as oans
from oracle import codec as ocodec
from oracle import levels as olevels
from oracle import rans_model as orm
from tests.golden_io import load_npz

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib():
    from latec_b200 import _lib

    return _lib


def test_library_exports_every_header_symbol():
    _l = _lib()
    lib = _l.load(require_gpu=False)
    header = open(os.path.join(ROOT, "include", "latec_b200.h")).read()
    names = set(re.findall(r"^\s*(?:const\s+)?(?:int|uint64_t|char\s*\*|const char\*)\s*\*?\s*(latec_\w+)\(",
                           header, re.M))
    names |= set(re.findall(r"\b(latec_\w+)\(", header))
    names = {n for n in names if not n.endswith("_t")}
    assert names, "no declarations found"
    for n in sorted(names):
        assert hasattr(lib, n), f"missing export {n}"
    assert set(names) == set(_l.SIGNATURES), "binding and header disagree"
    assert lib.latec_version().startswith(b"latec_b200")


def test_compute_entry_points_refuse_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(RuntimeError):
        _lib().load(require_gpu=True)


SCHEDULES = [((64, 64), 3, 8), ((33, 65), 4, 16), ((19, 23, 17), 3, 8), ((16, 16, 16, 16), 4, 16),
             ((17, 16, 16, 16, 16), 4, 16), ((64, 64), 5, 16), ((1, 7), 3, 8), ((5, 1, 7), 2, 4),
             ((9, 10, 11, 12), 2, 4), ((7, 5, 6, 3, 4, 5), 2, 4), ((2, 2), 4, 16), ((1, 1000), 5, 32)]


@pytest.mark.parametrize("shape,lv,stride", SCHEDULES)
def test_plan_counts_and_rank_decode_match_masks(shape, lv, stride):
    """The kernels' rank -> grid-index decode (run here on the host) visits
    every stage's points in the reference's flatnonzero(mask) order."""
    from latec_b200 import levels

    _l = _lib()
    lib = _l.load(require_gpu=False)
    p = levels.Plan(shape, lv, stride)
    assert p.counts == olevels.stage_counts(shape, lv, stride, 1)
    for t, m in enumerate(olevels.stage_masks(shape, lv, stride, 1)):
        want = np.flatnonzero(m)
        got = np.empty(len(want), np.int64)
        _l.check(lib.latec_plan_stage_flat(p.handle, t, 0, len(want), got.ctypes.data))
        assert np.array_equal(got, want), t


def test_plan_rejects_bad_parameters():
    from latec_b200 import levels

    with pytest.raises(ValueError):
        levels.Plan((64, 64), 3, 7)
    with pytest.raises(ValueError):
        levels.Plan((64, 64), 2, 16)
    with pytest.raises(ValueError):
        levels.Plan((), 2, 4)
    with pytest.raises(ValueError):
        levels.Plan((64, 64), 3, 8, 9)  # block larger than the anchor stride
    with pytest.raises(ValueError):
        levels.Plan((64, 64), 3, 8, 0)
    assert levels.Plan((64, 64), 3, 8, 4).counts[0] == 8 * 8 * 16  # 8 x 8 blocks of 4 x 4


def test_stage_ebs_match_reference_schedule():
    from latec_b200 import levels
    from tests.golden_io import schedule_cases

    for c in schedule_cases():
        got = levels.stage_ebs(tuple(c["shape"]), c["levels"], c["stride"], c["block"], 1e-3, 0.9)
        assert [float(v) for v in got] == c["ebs"]


def test_tables_match_reference_golden():
    from latec_b200 import rans_model as rm
    from tests.golden_io import sha

    z = load_npz("rans.npz")
    for t in z["meta"]["tables"]:
        assert sha(rm.cdfs(t["kexp"], t["shape"], t["owx"]).astype("<u4")) == t["sha"]
    for i, c in enumerate(z["meta"]["const_level"]):
        codes = z[f"cl_codes_{i}"]
        hist = orm.const_hist(codes, 1 << 15, c["kexp"])
        assert rm.fit_const_level(hist, len(codes), c["kexp"]) == (
            c["level"], c["shape"], c["owx"], c["bits"])


@pytest.mark.parametrize("n,kexp", [(5000, 3), (3 * (1 << 22) + 1234, 2), (9 * (1 << 22), 1),
                                    ((1 << 22) * 5 + 77, 9)])
def test_histogram_reconstruction_replays_float32_accumulation(n, kexp):
    """Per-segment window counts reproduce the reference's float32 histogram
    exactly, including bins whose count passes 2^24."""
    from latec_b200 import rans_model as rm

    rs = np.random.RandomState(n % 1000)
    span = (1 << kexp) - 1
    q = np.clip(np.round(rs.laplace(0, 0.05 if n > 1 << 24 else 2, n)), -span, span).astype(np.int64)
    codes = (q + (1 << 15)).astype(np.uint32)
    codes[rs.rand(n) < 1e-4] = 0
    want = orm.const_hist(codes, 1 << 15, kexp)
    nseg = -(-n // (1 << 22))
    seg = np.zeros((nseg, 2 * rm.HWIN), np.uint32)
    total = np.zeros(65536, np.uint32)
    for s in range(nseg):
        c = codes[s << 22:(s + 1) << 22]
        qq = c.astype(np.int64) - (1 << 15)
        inw = (c != 0) & (np.abs(qq) < rm.HWIN)
        seg[s] += np.bincount(np.where(c == 0, 0, np.where(inw, qq + rm.HWIN, 0)),
                              minlength=2 * rm.HWIN).astype(np.uint32) * 0
        seg[s, 0] = np.count_nonzero(c == 0)
        seg[s] += np.bincount(qq[inw] + rm.HWIN, minlength=2 * rm.HWIN).astype(np.uint32)
        big = (c != 0) & ~inw
        total += np.bincount(c[big], minlength=65536).astype(np.uint32)
    got = rm.stage_hist_f32(n, kexp, 1 << 15, seg, total)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_fast_quantisation_matches_oracle_c():
    from latec_b200 import rans_model as rm

    for kexp, shape, owx in [(1, 0, 0), (3, 5, 2), (8, 12, 7), (11, 20, 1)]:
        rows = rm.cdfs(kexp, shape, owx)
        got = rm.fast_quantize_rows(rows[::9])
        want = oans.wire_cdfs(rows[::9])
        assert np.array_equal(got, want)


def test_lanes_chunking_rule_matches_oracle():
    from latec_b200 import rans_model as rm

    for n, bits in [(1, 0.0), (100, 5.0), (65536, 3e3), (65536, 9e5), (50_000_000, 1e6),
                    (50_000_000, 2e8), (117_000_000, 5e9)]:
        assert rm.lanes_K(n, bits) == ocodec.lanes_K(n, bits)


def test_header_and_frame_layout_match_reference_format():
    from latec_b200 import bitstream as bs

    h = bs.Header(channels=1, src_dtype=1, spatial=(512, 512), eb=1e-3, levels=4,
                  anchor_stride=16, anchor_block=1, radius=1 << 15, max_radius=0, agg_level=-1,
                  vmin=-3.5, vmax=4.25, flags=bs.FLAG_INTERP | bs.FLAG_CUBIC | (1 << 9),
                  interp_center=0, eb_ratio=0.9)
    raw = h.pack()
    oh = ocodec.pack_header(dict(flags=h.flags, channels=1, src_dtype=1, levels=4,
                                 anchor_stride=16, anchor_block=1, interp_center=0,
                                 radius=1 << 15, eb=1e-3, vmin=-3.5, vmax=4.25, eb_ratio=0.9,
                                 spatial=(512, 512)))
    assert raw == oh and len(raw) == 80 + 1 + 8
    assert bs.Header.unpack(raw) == h
    with pytest.raises(ValueError):
        bs.Header.unpack(b"XXXXXXXX" + raw[8:])
    w = bs.pack_frame(12345, 7, 20, 63, 7, True)
    assert w == ocodec.framed(12345, 7, 20, 63, 7, True)
    assert bs.unpack_frame(w) == dict(hlen=12345, kexp=7, shape=20, level=63, owx=7, literal=True)
    with pytest.raises(ValueError):
        bs.pack_frame(1 << 45, 1, 0)


@pytest.mark.parametrize("n", [0, 1, 1000, 1 << 17, (1 << 17) + 1, 3 * (1 << 17), 700_001])
def test_raw_zstd_frame_is_a_valid_zstd_frame(n):
    from latec_b200 import bitstream as bs

    payload = np.random.RandomState(n % 97).randint(0, 256, n).astype(np.uint8)
    frame = bs.raw_zstd_frame(payload)
    assert bs.zstd().decompress_into(frame).tobytes() == payload.tobytes()
    assert bs.read_body(frame).tobytes() == payload.tobytes()
    assert frame.tobytes() == ocodec.raw_zstd_frame(payload.tobytes())
    z = bs.zstd().compress(payload.tobytes(), 3)
    assert bs.read_body(np.frombuffer(z, np.uint8)).tobytes() == payload.tobytes()


def test_level_thresholds_bracket_the_reference_levels():
    """The float32 level boundaries the device compares against reproduce
    latec/rans.py:270-278 exactly on both sides of every boundary."""
    from latec_b200.rans import level_thresholds
    from oracle import rans_model as orm

    for eb in (1e-6, 1e-3, 0.25, 3.0):
        th = level_thresholds(eb)
        assert th.dtype == np.float32 and np.all(np.diff(th) > 0)
        assert np.array_equal(orm.scale_to_level(th, eb), np.arange(1, 64))
        below = np.nextafter(th, np.float32(-np.inf))
        assert np.array_equal(orm.scale_to_level(below, eb), np.arange(0, 63))


def test_pick_shape_takes_the_first_least_total():
    """The shape choice's host half (latec_b200.rans.pick_shape): per
    candidate the fsum of its partial sums; the first least total wins."""
    import numpy as np

    from latec_b200 import rans

    P = rans._PARTIALS
    ids = [4, 7, 9]
    part = np.zeros((3, P))
    part[0, 0], part[1, 1], part[2, 2] = 5.0, 3.0, 3.0  # tie between the last two
    assert rans.pick_shape(ids, part.reshape(-1)) == 7
    part[2, 3] = -0.5
    assert rans.pick_shape(ids, part) == 9
    spread = np.full((3, P), 1.0)
    spread[1, -1] = 0.5  # the sum over all partials decides, not the first one
    assert rans.pick_shape(ids, spread) == 7


def test_plugin_stage_masks_are_the_reference_schedule():
    """The masks and point order a caller's predictor is given
    (latec_b200.codec._stage_flat) are the oracle schedule's masks in
    np.flatnonzero order, stage by stage."""
    import numpy as np

    from latec_b200 import levels
    from latec_b200.codec import _stage_flat
    from oracle import levels as olevels

    for shape, lv, st in [((40, 36), 2, 4), ((17, 20, 11), 2, 4), ((9, 8, 7, 6), 1, 2),
                          ((5, 130), 3, 8)]:
        plan = levels.plan_for(shape, lv, st, 1)
        want = list(olevels.iter_plan(shape, lv, st, 1))
        assert len(want) == len(plan)
        for t, (mask, _, _) in enumerate(want):
            assert np.array_equal(_stage_flat(plan, t), np.flatnonzero(mask))


def test_blocked_anchor_schedule_is_the_reference_schedule():
    """anchor_block > 1 (the anchors are anchor_block^ndim blocks on the anchor
    lattice and the finer stages skip those points, latec/levels.py:114-147):
    the plan's hole-aware rank -> point decode gives every stage's points in
    the oracle masks' flat order, for power-of-two and other block edges."""
    import numpy as np

    from latec_b200 import levels
    from latec_b200.codec import _stage_flat
    from oracle import levels as olevels

    for shape in [(37,), (19, 23), (9, 17, 20), (7, 9, 11, 6)]:
        for st, lv in [(4, 2), (8, 3), (8, 4)]:
            for block in (2, 3, 4, st):
                plan = levels.plan_for(shape, lv, st, block)
                masks = olevels.stage_masks(shape, lv, st, block)
                assert len(masks) == len(plan)
                for t, mask in enumerate(masks):
                    assert plan.counts[t] == int(mask.sum())
                    assert np.array_equal(_stage_flat(plan, t), np.flatnonzero(mask)), \
                        (shape, st, lv, block, t)


@pytest.mark.parametrize("radius,kexp", [(32768, 1), (32768, 7), (32768, 8), (32768, 15),
                                         (512, 9), (1, 1), (300, 8), (40000 // 2, 14)])
def test_literal_narrowing_matches_narrow(radius, kexp):
    """The literal stages' 16-bit narrowing equals the reference-form narrow()."""
    from latec_b200 import rans_model

    rng = np.random.default_rng(radius + kexp)
    span = 1 << kexp
    q = rng.integers(-(span - 1), span, 100000)
    codes = np.clip(q + radius, 1, 65535).astype(np.uint16)
    codes[rng.random(codes.size) < 0.05] = 0
    lo, hi = max(1, radius - span + 1), min(65535, radius + span - 1)
    codes[:4] = [0, lo, hi, radius]
    keep = (codes == 0) | ((codes.astype(np.int64) - radius >= -(span - 1))
                           & (codes.astype(np.int64) - radius <= span - 1))
    codes = codes[keep]
    want = rans_model.narrow(codes, radius, kexp).astype(rans_model.literal_dtype(kexp))
    got = rans_model.narrow_literals(codes, radius, kexp)
    assert got.dtype == want.dtype
    assert np.array_equal(got, want)


def test_trainer_rejects_unknown_precision():
    from latec_b200.train import Trainer

    with pytest.raises(ValueError):
        Trainer(precision="fp16")
