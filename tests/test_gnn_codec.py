"""The learned codec (latec/gnn_codec.py) on the device: the flat
dequantizer against the quantizer, and GNNCodec round trips with the bound
held on every value, deterministic streams and the reference container."""

import struct

import numpy as np
import pytest

RADIUS = 1 << 15


def test_auto_levels_follow_the_reference_table():
    from latec_b200.gnn_codec import auto_levels, per_step_eb_ratio

    assert auto_levels((512, 512), 1) == 8
    assert auto_levels((128, 128, 64, 64), 1) == 5
    assert auto_levels((256, 256, 256), 1) == 7
    assert auto_levels((256, 256, 256), 2) == 6
    assert auto_levels((20, 20), 1) == 3  # stride <= half the largest axis
    assert per_step_eb_ratio(0.9, 1) == 1.0
    assert per_step_eb_ratio(0.9, 5) ** 4 == pytest.approx(0.9)


def _field(shape, seed):
    rs = np.random.RandomState(seed)
    g = np.meshgrid(*[np.linspace(0, 1, n) for n in shape], indexing="ij")
    f = sum(np.sin((3 + k) * 2.7 * a + rs.rand() * 6) for k, a in enumerate(g))
    return (f + 0.02 * rs.randn(*shape)).astype(np.float32) * 7.0 - 3.0


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_flat_dequantize_matches_quantizer(dtype):
    import ctypes

    import torch

    from latec_b200 import _lib

    lib = _lib.load()
    ft = torch.float32 if dtype == "f32" else torch.float64
    rs = np.random.RandomState(4)
    n = 300_001
    x = torch.from_numpy(rs.randn(n) * 5).to(ft).cuda()
    pred = (x + torch.from_numpy(rs.randn(n) * 0.01).to(ft).cuda()).contiguous()
    x[::101] = 1e6
    prm = _lib.QuantParams(dtype=_lib.F32 if dtype == "f32" else _lib.F64, channels=1,
                           radius=RADIUS, order=1, center=0, end_mode=1, round_output=0,
                           reserved=0)
    codes = torch.empty(n, dtype=torch.int16, device="cuda")
    recon = torch.empty(n, dtype=ft, device="cuda")
    outl = torch.empty(n, dtype=ft, device="cuda")
    stats = torch.zeros(ctypes.sizeof(_lib.StageStats), dtype=torch.uint8, device="cuda")
    hseg = torch.empty(512, dtype=torch.int32, device="cuda")
    htot = torch.empty(65536, dtype=torch.int32, device="cuda")
    ws = torch.empty(int(lib.latec_flat_workspace_bytes(n, prm.dtype)), dtype=torch.uint8,
                     device="cuda")
    sp = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.latec_quantize(ctypes.byref(prm), 0.01, n, x.data_ptr(), pred.data_ptr(),
                                  codes.data_ptr(), recon.data_ptr(), outl.data_ptr(),
                                  stats.data_ptr(), hseg.data_ptr(), htot.data_ptr(),
                                  ws.data_ptr(), ws.numel(), sp))
    st = _lib.StageStats.from_buffer_copy(stats.cpu().numpy().tobytes())
    assert st.n_out > n // 101 - 2
    back = torch.full((n,), 7.0, dtype=ft, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws2 = torch.empty(int(lib.latec_dequantize_workspace_bytes(n)), dtype=torch.uint8,
                      device="cuda")
    _lib.check(lib.latec_dequantize(ctypes.byref(prm), 0.01, n, pred.data_ptr(), codes.data_ptr(),
                                    outl.data_ptr(), st.n_out, back.data_ptr(), err.data_ptr(),
                                    ws2.data_ptr(), ws2.numel(), sp))
    assert int(err.item()) == 0
    assert torch.equal(back.view(torch.uint8), recon.view(torch.uint8))
    _lib.check(lib.latec_dequantize(ctypes.byref(prm), 0.01, n, pred.data_ptr(), codes.data_ptr(),
                                    outl.data_ptr(), st.n_out - 1, back.data_ptr(),
                                    err.data_ptr(), ws2.data_ptr(), ws2.numel(), sp))
    assert int(err.item()) & 1


def _codec(seed=7, agg=1):
    from latec_b200 import gnn
    from latec_b200.gnn_codec import GNNCodec

    return GNNCodec(weights=gnn.random_weights(seed, 64, agg), d=64, agg_level=agg)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,levels,eb,tune,fp16", [((40, 36), 3, 1e-3, "fast", True),
                                                        ((40, 36), 3, 1e-3, "fast", False),
                                                        ((24, 20, 18), 2, 1e-2, "size", True),
                                                        ((70, 9), "auto", 3e-3, "fast", True)])
def test_gnn_codec_round_trip_holds_the_bound(shape, levels, eb, tune, fp16):
    import torch

    from latec_b200.gnn_codec import MAGIC, VERSION, read_stream

    codec = _codec()
    x = _field(shape, 3)
    s1 = codec.compress(x, eb, levels=levels, tune=tune, fp16=fp16)
    s2 = codec.compress(torch.from_numpy(x).cuda(), eb, levels=levels, tune=tune, fp16=fp16)
    assert s1 == s2  # deterministic, host or device input
    magic, version, hlen = struct.unpack_from("<8sII", s1, 0)
    assert magic == MAGIC and version == VERSION
    meta, _ = read_stream(s1)
    assert meta["shape"] == list(shape) and meta["dtype"] == np.dtype(np.float32).str
    assert meta["fp16"] == fp16 and meta["float_path"].startswith("latec_b200-")
    out = codec.uncompress(s1)
    assert isinstance(out, torch.Tensor) and out.dtype == torch.float32
    assert tuple(out.shape) == shape
    vmin, vmax = float(np.float32(x.min())), float(np.float32(x.max()))
    xn = (x.astype(np.float32) - np.float32(vmin)) / np.float32(vmax - vmin)
    on = (out.numpy() - np.float32(vmin)) / np.float32(vmax - vmin)
    slack = 4 * np.finfo(np.float32).eps
    assert np.abs(on.astype(np.float64) - xn).max() <= eb + slack
    assert np.array_equal(codec.uncompress(s1).numpy(), out.numpy())
    assert len(s1) < x.nbytes


@pytest.mark.gpu
def test_gnn_codec_float64_and_errors():
    import torch

    from latec_b200.gnn_codec import GNNCodec

    codec = _codec()
    x = _field((33, 31), 5).astype(np.float64)
    s = codec.compress(x, 1e-3, levels=3)
    out = codec.uncompress(s)
    assert out.dtype == torch.float64
    span = x.max() - x.min()
    assert np.abs(out.numpy() - x).max() <= 1e-3 * span * (1 + 1e-5) + 1e-6 * span
    with pytest.raises(ValueError):
        codec.uncompress(b"NOTLATEC" + s[8:])
    with pytest.raises(ValueError):
        _codec(seed=8).uncompress(s)  # foreign weights: checkpoint hash differs
    assert _codec(seed=8).__class__ is GNNCodec
    with pytest.raises(ValueError):
        codec.compress(np.zeros((0, 4), np.float32), 1e-3)
    with pytest.raises(ValueError):
        codec.compress(x, 0.0)
    with pytest.raises(ValueError):
        codec.compress(x, 1e-3, levels=3, chunk_size=12)  # not a multiple of the stride
    with pytest.raises(FileNotFoundError):
        GNNCodec("/nonexistent/checkpoint.pt")


@pytest.mark.gpu
@pytest.mark.parametrize("shape,levels", [((64, 60), 4), ((24, 22, 20), 3), ((12, 12, 10, 10), 2)])
def test_gate_falls_back_to_interpolation_where_it_codes_fewer_bits(shape, levels):
    from latec_b200.gnn_codec import gate_fields, read_stream, unpack_gates

    codec = _codec()  # untrained weights: interpolation wins on a smooth field
    x = _field(shape, 9)
    gated = codec.compress(x, 1e-3, levels=levels)
    plain = codec.compress(x, 1e-3, levels=levels, gate=False)
    meta, _ = read_stream(gated)
    words = unpack_gates(meta["gates"])
    assert gate_fields(words[0])[0] == 0  # the anchors have no interpolation
    assert any(gate_fields(w)[0] for w in words)  # some stage fell back
    assert all(w == 0 for w in unpack_gates(read_stream(plain)[0]["gates"]))
    assert len(gated) < len(plain)
    assert codec.compress(x, 1e-3, levels=levels) == gated  # deterministic
    out = codec.uncompress(gated).numpy()
    vmin, vmax = float(np.float32(x.min())), float(np.float32(x.max()))
    xn = (x.astype(np.float32) - np.float32(vmin)) / np.float32(vmax - vmin)
    on = (out - np.float32(vmin)) / np.float32(vmax - vmin)
    assert np.abs(on.astype(np.float64) - xn).max() <= 1e-3 + 4 * np.finfo(np.float32).eps
    assert np.array_equal(codec.uncompress(gated).numpy(), out)


@pytest.mark.gpu
def test_device_gate_choice_follows_the_host_rule():
    """latec_gate_choose_apply's word equals gate_word(*gate_choose(sums)) on
    random rate tables and on ones built to take each branch."""
    import torch

    from latec_b200 import _lib
    from latec_b200.gnn_codec import GATE_SHIFTS, GATE_T, gate_choose, gate_fields, gate_word

    lib = _lib.load()
    R, NB = 1 + 3 * len(GATE_SHIFTS), len(GATE_T) + 1
    rs = np.random.RandomState(5)
    cases = [np.zeros((R, NB), np.int64)]
    low = np.full((R, NB), 1000, np.int64)
    low[5, :4] = 10  # a candidate cheaper only in the low buckets
    high = np.full((R, NB), 1000, np.int64)
    high[9, 8:] = 10  # and one cheaper only in the high buckets
    cases += [low, high]
    for _ in range(300):
        t = rs.randint(0, 1 << 30, size=(R, NB)).astype(np.int64)
        if rs.rand() < 0.8:
            r, c = rs.randint(1, R), rs.randint(0, NB)
            t[r, c:] //= rs.randint(2, 50)
        cases.append(t)
    word = torch.zeros(1, dtype=torch.int32, device="cuda")
    kinds, dirs = set(), set()
    for sums in cases:
        dev_sums = torch.from_numpy(sums.reshape(-1)).cuda()
        _lib.check(lib.latec_gate_choose_apply(0, dev_sums.data_ptr(), None, None, None, None,
                                               None, 1e-3, word.data_ptr(), _lib.stream_ptr()))
        want = gate_word(*gate_choose(sums))
        got = int(word.item())
        assert got == want, (got, want)
        kind, direction, _, _ = gate_fields(got)
        kinds.add(kind)
        if kind:
            dirs.add(direction)
    assert kinds == {0, 1, 2, 3} and dirs == {0, 1}


@pytest.mark.gpu
@pytest.mark.parametrize("shape,levels,chunk", [((64, 60), 4, None), ((24, 22, 20), 3, None),
                                                ((40, 36), 2, 16)])
def test_gate_fine_shares_one_word_over_the_finest_level(shape, levels, chunk):
    from latec_b200.gnn_codec import (chunk_edges, chunk_groups, pack_gates, read_stream,
                                      unpack_gates, write_stream)
    from latec_b200.levels import stage_counts, stage_strides

    codec = _codec()
    x = _field(shape, 9)
    fine = codec.compress(x, 1e-3, levels=levels, gate_fine=True, chunk_size=chunk)
    per = codec.compress(x, 1e-3, levels=levels, chunk_size=chunk)
    (mf, payload), mp = read_stream(fine), read_stream(per)[0]
    assert mf["gate_fine"] and not mp["gate_fine"] and "fine_gates" not in mp
    # the per-stage stream's words, cut into batches; its finest words give way
    # to the first of them in the shared-word stream
    stride = 1 << levels
    edges = chunk_edges(shape, stride, chunk) or shape
    cb = mf.get("chunk_batch", 1)
    wp, want_gates, want_fine = unpack_gates(mp["gates"]), [], []
    for cshape, origins in chunk_groups(shape, edges):
        counts = stage_counts(cshape, levels, stride)
        strides = stage_strides(len(shape), levels, stride)
        finest = [s == 1 for s, n in zip(strides, counts) if n]
        for _ in range(0, len(origins), cb):
            ws, wp = wp[:len(finest)], wp[len(finest):]
            want_gates += [w for w, f in zip(ws, finest) if not f]
            want_fine += [w for w, f in zip(ws, finest) if f][:1]
    assert not wp
    assert unpack_gates(mf["gates"]) == want_gates
    assert unpack_gates(mf["fine_gates"]) == want_fine
    assert codec.compress(x, 1e-3, levels=levels, gate_fine=True, chunk_size=chunk) == fine
    out = codec.uncompress(fine).numpy()
    vmin, vmax = float(np.float32(x.min())), float(np.float32(x.max()))
    xn = (x.astype(np.float32) - np.float32(vmin)) / np.float32(vmax - vmin)
    on = (out - np.float32(vmin)) / np.float32(vmax - vmin)
    assert np.abs(on.astype(np.float64) - xn).max() <= 1e-3 + 4 * np.finfo(np.float32).eps
    # without the gate there is nothing to share
    off = read_stream(codec.compress(x, 1e-3, levels=levels, gate=False, gate_fine=True,
                                     chunk_size=chunk))[0]
    assert not off["gate_fine"] and "fine_gates" not in off
    # a finest word short is a malformed stream
    bad = dict(mf, fine_gates=pack_gates(unpack_gates(mf["fine_gates"])[:-1]))
    with pytest.raises(ValueError):
        codec.uncompress(write_stream(bad, payload, 3))


@pytest.mark.gpu
@pytest.mark.parametrize("predictor,order,center", [("interp-cubic", "cubic", 0),
                                                    ("interp-linear", "linear", 1),
                                                    ("interp-linear-last", "linear", 2)])
@pytest.mark.parametrize("shape,levels", [((40, 36), 3), ((24, 22, 20), 3)])
def test_interpolation_ablation_reconstructs_as_the_plain_codec(predictor, order, center, shape,
                                                                levels):
    """The ablation codes every stage against the gate's interpolation
    candidate (anchors against 0), so on the normalised field its
    reconstruction is the plain codec's with that predictor, bit for bit."""
    import torch

    import latec_b200 as lb
    from latec_b200.gnn_codec import (EB_COARSE_FACTOR, GATE_END_MODE, per_step_eb_ratio,
                                      read_stream, unpack_gates)

    codec = _codec()
    x = _field(shape, 13)
    s = codec.compress(x, 1e-3, levels=levels, predictor=predictor)
    meta, _ = read_stream(s)
    assert meta["predictor"] == predictor and not meta["gate"]
    assert not any(unpack_gates(meta["gates"]))
    assert codec.compress(x, 1e-3, levels=levels, predictor=predictor) == s
    out = codec.uncompress(s)
    vmin, vmax = float(np.float32(x.min())), float(np.float32(x.max()))
    span = vmax - vmin
    xn = ((torch.from_numpy(x).cuda() - np.float32(vmin)) / np.float32(span)).contiguous()
    stride = 1 << levels
    pred = lb.InterpPredictor(order, levels, stride, 1, center=center, end_mode=GATE_END_MODE)
    _, st = lb.compress(xn, 1e-3, pred, levels=levels, anchor_stride=stride,
                        eb_ratio=per_step_eb_ratio(EB_COARSE_FACTOR, levels), recon="device")
    want = st["recon"].reshape(shape) * np.float32(span) + np.float32(vmin)
    assert torch.equal(out.cuda(), want)
    gnn_s = codec.compress(x, 1e-3, levels=levels)
    assert read_stream(gnn_s)[0]["predictor"] == "gnn"
    with pytest.raises(ValueError):
        codec.compress(x, 1e-3, levels=levels, predictor="interp-quintic")


@pytest.mark.gpu
def test_interpolation_ablation_on_a_chunk_grid():
    from latec_b200.gnn_codec import read_stream

    codec = _codec()
    x = _field((70, 66), 14)
    s = codec.compress(x, 1e-3, levels=3, chunk_size=16, predictor="interp-cubic")
    assert read_stream(s)[0]["chunk_batch"] >= 1
    out = codec.uncompress(s).numpy()
    vmin, vmax = float(np.float32(x.min())), float(np.float32(x.max()))
    xn = (x.astype(np.float32) - np.float32(vmin)) / np.float32(vmax - vmin)
    on = (out - np.float32(vmin)) / np.float32(vmax - vmin)
    assert np.abs(on.astype(np.float64) - xn).max() <= 1e-3 + 4 * np.finfo(np.float32).eps


@pytest.mark.gpu
def test_fp8_float_path_round_trip():
    from latec_b200.gnn_codec import FLOAT_PATHS, read_stream

    codec = _codec()
    x = _field((40, 36), 4)
    s = codec.compress(x, 1e-3, levels=3, fp8=True)
    assert read_stream(s)[0]["float_path"] == FLOAT_PATHS["fp8"]
    assert codec.compress(x, 1e-3, levels=3, fp8=True) == s
    out = codec.uncompress(s).numpy()
    vmin, vmax = float(np.float32(x.min())), float(np.float32(x.max()))
    xn = (x.astype(np.float32) - np.float32(vmin)) / np.float32(vmax - vmin)
    on = (out - np.float32(vmin)) / np.float32(vmax - vmin)
    assert np.abs(on.astype(np.float64) - xn).max() <= 1e-3 + 4 * np.finfo(np.float32).eps
    with pytest.raises(ValueError):
        codec.compress(x, 1e-3, levels=3, fp8=True, fp16=False)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.int16, np.int32, np.uint8, np.bool_])
def test_integer_sources_round_trip(dtype):
    import torch

    codec = _codec()
    f = _field((36, 34), 6)
    if dtype == np.bool_:
        x = f > np.median(f)
    elif dtype == np.uint8:
        x = np.clip((f - f.min()) / (f.max() - f.min()) * 255, 0, 255).round().astype(np.uint8)
    else:
        x = np.round(f * 900).astype(dtype)
    eb = 2e-3
    s = codec.compress(x, eb, levels=3)
    out = codec.uncompress(s)
    assert out.dtype == getattr(torch, np.dtype(dtype).name) and tuple(out.shape) == x.shape
    o = out.numpy()
    if dtype == np.bool_:
        assert np.array_equal(o, x)  # a bound below 0.5 of the range keeps every bool
        return
    span = float(np.float32(x.max())) - float(np.float32(x.min()))
    err = np.abs(o.astype(np.float64) - x.astype(np.float64)).max()
    # signed integers: the bound is checked on the returned integer itself;
    # unsigned ones (as in the reference) only on the float reconstruction
    limit = eb * span * (1 + 1e-5) + (0.0 if np.dtype(dtype).kind == "i" else 0.5)
    assert err <= limit, (err, limit)


@pytest.mark.gpu
def test_flat_quantizer_checks_the_raw_integer():
    """round_output 2 against a NumPy restatement of _quantize_t's (span,
    offset) check (latec/gnn_codec.py:998-1031)."""
    import ctypes

    import torch

    from latec_b200 import _lib

    lib = _lib.load()
    rs = np.random.RandomState(9)
    n = 200_000
    span, off = 1234.0, -17.0
    raw = rs.randint(-17, 1217, n).astype(np.float64)
    x = ((raw - off) / span).astype(np.float32)
    pred = (x + rs.randn(n).astype(np.float32) * 3e-3).astype(np.float32)
    # above half a raw unit (0.5 / 1234 in normalised terms): the nearest raw
    # integer of a reconstruction can be the wrong one, and the check rejects it
    eb = 7e-4
    prm = _lib.QuantParams(dtype=_lib.F32, channels=1, radius=RADIUS, order=1, center=0,
                           end_mode=1, round_output=2, reserved=0, round_span=span,
                           round_offset=off)
    xd, pd = torch.from_numpy(x).cuda(), torch.from_numpy(pred).cuda()
    codes = torch.empty(n, dtype=torch.int16, device="cuda")
    recon = torch.empty(n, dtype=torch.float32, device="cuda")
    outl = torch.empty(n, dtype=torch.float32, device="cuda")
    stats = torch.zeros(ctypes.sizeof(_lib.StageStats), dtype=torch.uint8, device="cuda")
    hseg = torch.empty(512, dtype=torch.int32, device="cuda")
    htot = torch.empty(65536, dtype=torch.int32, device="cuda")
    ws = torch.empty(int(lib.latec_flat_workspace_bytes(n, _lib.F32)), dtype=torch.uint8,
                     device="cuda")
    _lib.check(lib.latec_quantize(ctypes.byref(prm), eb, n, xd.data_ptr(), pd.data_ptr(),
                                  codes.data_ptr(), recon.data_ptr(), outl.data_ptr(),
                                  stats.data_ptr(), hseg.data_ptr(), htot.data_ptr(),
                                  ws.data_ptr(), ws.numel(), torch.cuda.current_stream().cuda_stream))
    got = codes.cpu().numpy().view(np.uint16).astype(np.int64)
    w = 2.0 * eb
    q = np.rint((x.astype(np.float64) - pred.astype(np.float64)) / w).astype(np.int64)
    inr = np.abs(q) < RADIUS
    cand = np.where(inr, q + RADIUS, 0)
    rc = (pred.astype(np.float64) + w * (cand - RADIUS)).astype(np.float32)
    chk = ((np.rint(rc.astype(np.float64) * span + off) - off) / span).astype(np.float32)
    ok = inr & (np.abs(x - chk) <= np.float32(eb))
    want = np.where(ok, cand, 0)
    assert np.array_equal(got, want)
    assert 0 < (want == 0).sum() < n  # the check rejects some, keeps most


def test_chunk_grid_on_host():
    """The automatic edges of the reference's rule, and a grid that covers every
    point exactly once, chunks grouped by shape in raster order."""
    from latec_b200.gnn_codec import (AUTO_CHUNK_THRESHOLD, auto_chunk_edges, chunk_edges,
                                      chunk_groups)

    assert auto_chunk_edges((128, 128, 64, 64), 32) == (32, 32, 32, 32)
    assert chunk_edges((128, 128, 64, 64), 32, None) == (32, 32, 32, 32)
    assert chunk_edges((64, 64), 16, None) is None  # below the budget: one region
    assert chunk_edges((64, 64), 16, 64) is None
    assert chunk_edges((64, 64), 16, (32, 16)) == (32, 16)
    e = auto_chunk_edges((4000, 3), 8)
    assert e[1] == 8 and e[0] % 8 == 0 and e[0] * 3 <= 2 * AUTO_CHUNK_THRESHOLD
    for shape, edges in (((70, 66), (16, 16)), ((9, 40, 33), (8, 16, 8))):
        seen = np.zeros(shape, np.int32)
        for cshape, origins in chunk_groups(shape, edges):
            for o in origins:
                assert tuple(min(e, n - a) for e, n, a in zip(edges, shape, o)) == cshape
                seen[tuple(slice(a, a + c) for a, c in zip(o, cshape))] += 1
        assert np.all(seen == 1)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,levels,chunk", [((70, 66), 3, 16), ((24, 40, 18), 2, (8, 16, 8))])
def test_chunked_round_trip_holds_the_bound(shape, levels, chunk):
    from latec_b200.gnn_codec import read_stream

    codec = _codec()
    x = _field(shape, 11)
    s = codec.compress(x, 1e-3, levels=levels, chunk_size=chunk)
    meta, _ = read_stream(s)
    assert meta["chunk_batch"] >= 1 and meta["chunks"] == list(
        (chunk,) * len(shape) if np.isscalar(chunk) else chunk)
    assert codec.compress(x, 1e-3, levels=levels, chunk_size=chunk) == s  # deterministic
    out = codec.uncompress(s).numpy()
    vmin, vmax = float(np.float32(x.min())), float(np.float32(x.max()))
    xn = (x.astype(np.float32) - np.float32(vmin)) / np.float32(vmax - vmin)
    on = (out - np.float32(vmin)) / np.float32(vmax - vmin)
    assert np.abs(on.astype(np.float64) - xn).max() <= 1e-3 + 4 * np.finfo(np.float32).eps
    one = codec.compress(x, 1e-3, levels=levels)  # the same tensor as one region
    assert "chunk_batch" not in read_stream(one)[0]
