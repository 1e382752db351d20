"""GPU parity of the plain codec against the CPU oracle and the reference's golden vectors.

Every test here runs the CUDA library through its C ABI (via the Python host
package) and checks results bit for bit: per-stage codes and outliers in scan
order, the reconstruction, and the stream bytes of both entropy modes.
"""

import numpy as np
import pytest

from oracle import codec as ocodec
from tests.golden_io import codec_case_names, load_npz, sha

pytestmark = pytest.mark.gpu


def _lb():
    import latec_b200

    return latec_b200


def _field_for(name, z):
    if "x" in z:
        return z["x"]
    from latec_b200 import fields

    if name == "cfg1_512x512":
        return fields.grf_se((512, 512), 16.0, seed=0)
    return fields.turbulence_jumps((64, 64, 64), seed=6)


def _gpu_compress(x, m, entropy="native"):
    lb = _lb()
    pk, ck = m["predictor"], m["compress"]
    pred = lb.InterpPredictor(m["order"], ck["levels"], ck["anchor_stride"], ck["anchor_block"],
                              center=pk.get("center"), end_mode=pk.get("end_mode"))
    return lb.compress(x, m["eb"], pred, levels=ck["levels"], anchor_stride=ck["anchor_stride"],
                       anchor_block=ck["anchor_block"], radius=ck.get("radius", 1 << 15),
                       eb_ratio=ck.get("eb_ratio"), entropy=entropy)


def _bytes(a):
    return np.ascontiguousarray(np.asarray(a)).view(np.uint8)


def _oracle_stages(stream):
    """Stage codes / outliers of a stream, parsed and entropy-decoded by the oracle."""
    h = ocodec.unpack_header(stream)
    payload = ocodec.zstd().decompress(stream[h["body_offset"]:])
    mode = "native" if h["flags"] & ocodec.FLAG_LANES else "compat"
    ft = np.float64 if h["src_dtype"] == 2 else np.float32
    from oracle import levels as olv

    ns = olv.n_stages(len(h["spatial"]), h["levels"])
    off, out = 0, []
    for _ in range(ns):
        codes, outl, off = ocodec.unpack_stage(payload, off, h["radius"], mode, ft)
        out.append((codes, outl))
    assert off == len(payload)
    return out


@pytest.mark.parametrize("name", codec_case_names())
def test_stage_codes_outliers_recon_bit_exact(name):
    z = load_npz(f"codec_{name}.npz")
    m = z["meta"]
    x = _field_for(name, z)
    stream, st = _gpu_compress(x, m)
    assert (st["interp_center"], st["interp_end_mode"], st["eb_ratio"]) == (
        m["center"], m["end_mode"], m["eb_ratio"])
    stages = _oracle_stages(stream)
    assert len(stages) == len(m["stages"])
    for t, ((codes, outl), want) in enumerate(zip(stages, m["stages"])):
        assert sha(codes.astype("<u4")) == want["codes_sha"], f"stage {t} codes"
        assert sha(np.asarray(outl, np.float32).astype("<f4")) == want["out_sha"], f"stage {t} outliers"
    assert st["stage_outliers"] == m["stage_outliers"]
    assert sha(np.asarray(st["recon"], np.float32).astype("<f4")) == m["recon_sha"]
    back = _lb().decompress(stream)
    assert np.array_equal(_bytes(back), _bytes(st["recon"]))


@pytest.mark.parametrize("name", ["grf2d_128", "odd3d_c0_e1", "odd3d_c2_e3", "grf4d_default_center",
                                  "block4_3d", "block3_2d_linear",
                                  "nan_inf_2d", "small_radius", "image_3ch", "turb3d_64_rel1e-4",
                                  "cfg1_512x512", "thin_17x1x9", "tiny_2x2"])
@pytest.mark.parametrize("entropy", ["native", "compat"])
def test_stream_bytes_match_oracle(name, entropy):
    """The whole stream -- model fits, lane chunking, rANS words, records -- is
    byte-identical to the oracle's for the same input and mode."""
    z = load_npz(f"codec_{name}.npz")
    m = z["meta"]
    x = _field_for(name, z)
    stream, st = _gpu_compress(x, m, entropy)
    pk, ck = m["predictor"], m["compress"]
    ostream, ost = ocodec.compress(
        x, m["eb"], order=m["order"], levels_=ck["levels"], anchor_stride=ck["anchor_stride"],
        anchor_block=ck["anchor_block"], radius=ck.get("radius", 1 << 15),
        eb_ratio=ck.get("eb_ratio"), center=pk.get("center"), end_mode=pk.get("end_mode"),
        mode=entropy)
    gh, oh = ocodec.unpack_header(stream), ocodec.unpack_header(ostream)
    assert stream[:gh["body_offset"]] == ostream[:oh["body_offset"]]
    gp = ocodec.zstd().decompress(stream[gh["body_offset"]:])
    op = ocodec.zstd().decompress(ostream[oh["body_offset"]:])
    assert gp == op
    if entropy == "native":
        assert stream == ostream
    # cross decode: the oracle reads the GPU stream and the GPU reads the oracle's
    back_o = ocodec.decompress(stream)
    assert np.array_equal(_bytes(back_o), _bytes(st["recon"]))
    back_g = _lb().decompress(ostream)
    assert np.array_equal(_bytes(back_g), _bytes(ost["recon"]))


def test_float64_path_matches_oracle_and_bound():
    from latec_b200 import fields

    x = fields.turbulence_jumps((40, 36, 30), seed=21).astype(np.float64) * 1e3
    eb = 1e-6
    lb = _lb()
    stream, st = lb.compress(x, eb, lb.InterpPredictor("cubic", 3, 8, 1), levels=3, anchor_stride=8)
    ostream, ost = ocodec.compress(x, eb, levels_=3, anchor_stride=8, mode="native")
    assert stream == ostream
    back = lb.decompress(stream)
    assert back.dtype == np.float64
    assert np.array_equal(back, ost["recon"])
    assert np.abs(back - x).max() <= eb


def test_uint8_image_round_output():
    rs = np.random.RandomState(3)
    img = (np.clip(rs.rand(60, 75, 3) * 40 + np.linspace(0, 200, 75)[None, :, None], 0, 255)).astype(np.uint8)
    lb = _lb()
    for eb in (0.5, 2.0, 1.5):
        stream, st = lb.compress(img, eb, lb.InterpPredictor("cubic", 3, 8, 1), levels=3,
                                 anchor_stride=8)
        ostream, ost = ocodec.compress(img, eb, levels_=3, anchor_stride=8, mode="native")
        assert stream == ostream
        back = lb.decompress(stream)
        assert back.dtype == np.uint8 and np.array_equal(back, ost["recon"])
        assert np.abs(back.astype(np.int64) - img).max() <= eb


def test_predict_api_matches_reference_predictions():
    from oracle import levels as olv

    z = load_npz("predict.npz")
    lb = _lb()
    recon = z["recon2d"]
    shape = recon.shape[1:]
    for order in ("linear", "cubic"):
        for center in (0, 1, 2):
            for em in (0, 1, 2, 3):
                p = lb.InterpPredictor(order, 3, 8, 1, center=center, end_mode=em)
                known = np.zeros(shape, bool)
                for t, (mask, s, axes) in enumerate(olv.iter_plan(shape, 3, 8, 1)):
                    key = f"p2d_{order}_{center}_{em}_{t}"
                    if key in z:
                        got = p.predict(recon, known, mask)
                        assert np.array_equal(got, z[key]), key
                    known |= mask


def test_cfg1_full_size_bound_and_roundtrip():
    """512^2 GRF at eb 1e-3 (the CPU-runnable workload), both modes."""
    from latec_b200 import fields

    x = fields.grf_se((512, 512), 16.0, seed=0)
    lb = _lb()
    for entropy in ("native", "compat"):
        stream, st = lb.compress(x, 1e-3, lb.InterpPredictor("cubic", 4, 16, 1), entropy=entropy)
        back = lb.decompress(stream)
        assert np.abs(back.astype(np.float64) - x).max() <= 1e-3
        assert np.array_equal(back, st["recon"])


@pytest.mark.parametrize("shape,lv,stride", [((160, 130, 100), 5, 32), ((8, 300, 7, 9), 3, 8),
                                             ((3, 5, 4, 6, 2, 5), 2, 4)])
def test_larger_and_high_rank_fields_match_oracle(shape, lv, stride):
    from latec_b200 import fields

    x = fields.turbulence_jumps(shape, seed=9)
    eb = 1e-3 * float(x.max() - x.min())
    lb = _lb()
    stream, st = lb.compress(x, eb, lb.InterpPredictor("cubic", lv, stride, 1), levels=lv,
                             anchor_stride=stride)
    ostream, _ = ocodec.compress(x, eb, levels_=lv, anchor_stride=stride, mode="native")
    assert stream == ostream
    back = lb.decompress(stream)
    assert np.abs(back.astype(np.float64) - x).max() <= eb


@pytest.mark.parametrize("tile_mode", [0, 2])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_256cube_stream_matches_oracle(dtype, tile_mode):
    """256^3 turbulence + jumps at rel eb 1e-4 (cubic, levels 6, stride 64):
    the benchmark's schedule at a size the CPU oracle codes in seconds, so the
    stream (native mode) and reconstruction are compared byte for byte with
    the oracle's, with per-stage launches (tile mode 0, the default) and with
    the fused level kernels (mode 2); float64 is the FP64 bound path."""
    from latec_b200 import _lib, fields

    x = fields.turbulence_jumps((256, 256, 256), seed=2).astype(dtype)
    eb = 1e-4 * float(np.float64(x.max()) - np.float64(x.min()))
    lb = _lb()
    lib = _lib.load()
    _lib.check(lib.latec_set_tile_mode(tile_mode))
    try:
        stream, st = lb.compress(x, eb, lb.InterpPredictor("cubic", 6, 64, 1), levels=6,
                                 anchor_stride=64)
        back = lb.decompress(stream)
    finally:
        _lib.check(lib.latec_set_tile_mode(0))
    ostream, ost = ocodec.compress(x, eb, levels_=6, anchor_stride=64, mode="native")
    assert stream == ostream
    assert np.array_equal(back, ost["recon"])
    assert np.abs(back.astype(np.float64) - x.astype(np.float64)).max() <= eb


@pytest.mark.parametrize("shape,dtype,order,center", [
    ((256, 256, 256), np.float32, "cubic", 0),
    ((130, 300, 257), np.float32, "cubic", 0),
    ((64, 96, 160), np.float64, "cubic", 0),
    ((200, 1030), np.float32, "cubic", 0),
    ((24, 40, 20, 300), np.float32, "cubic", 1),
    ((90, 70, 260), np.float32, "linear", 2),
])
def test_row_segments_match_per_point_decode(shape, dtype, order, center):
    """The row-segment stage kernels (the default) and the per-point decode
    code the same stream and reconstruction, rows of every length and parity: ragged
    last axes, float64, rank 2 and 4, linear order, both single-axis centers;
    the stream of the first case is also the oracle's."""
    from latec_b200 import _lib, fields

    x = fields.turbulence_jumps(shape, seed=3).astype(dtype)
    eb = 1e-4 * float(np.float64(x.max()) - np.float64(x.min()))
    lb = _lb()
    lib = _lib.load()
    lv = 4 if len(shape) == 4 else 5
    pred = lambda: lb.InterpPredictor(order, lv, 16, 1, center=center)  # noqa: E731
    got = {}
    try:
        for mode in (1, 0):
            _lib.check(lib.latec_set_row_mode(mode))
            got[mode] = lb.compress(x, eb, pred(), levels=lv, anchor_stride=16)
        _lib.check(lib.latec_set_row_mode(1))
        back = lb.decompress(got[1][0])  # decoded with row segments
    finally:
        _lib.check(lib.latec_set_row_mode(1))
    assert got[1][0] == got[0][0]
    assert np.array_equal(back, got[0][1]["recon"])
    assert np.array_equal(got[1][1]["recon"], got[0][1]["recon"])
    if shape == (256, 256, 256):
        ostream, _ = ocodec.compress(x, eb, levels_=lv, anchor_stride=16, mode="native")
        assert got[1][0] == ostream


def test_full_size_512cube_properties():
    """512^3 float32 turbulence + jumps at rel eb 1e-4 (the benchmark workload):
    bound, encoder recon == decoder output, determinism of two encodes."""
    import torch

    from latec_b200 import fields

    x = fields.turbulence_jumps((512, 512, 512), seed=0, device="cuda")
    mm = torch.aminmax(x)
    eb = 1e-4 * (float(mm.max.item()) - float(mm.min.item()))
    lb = _lb()
    pred = lb.InterpPredictor("cubic", 6, 64, 1)
    s1, st1 = lb.compress(x, eb, pred, levels=6, anchor_stride=64)
    s2, _ = lb.compress(x, eb, lb.InterpPredictor("cubic", 6, 64, 1), levels=6, anchor_stride=64)
    assert s1 == s2
    back = lb.decompress(s1, out="device")
    assert torch.equal(back, st1["recon"])
    assert float((back.double() - x.double()).abs().max().item()) <= eb
    del x, back


def test_tune_size_sweep_runs_and_picks_smallest():
    from latec_b200 import fields

    x = fields.turbulence_jumps((48, 40, 36), seed=5)
    lb = _lb()
    stream, st = lb.compress(x, 1e-3, lb.InterpPredictor("cubic", 3, 8, 1), levels=3,
                             anchor_stride=8, tune="size")
    assert st["tune_candidates"] > 1
    back = lb.decompress(stream)
    assert np.abs(back.astype(np.float64) - x).max() <= 1e-3


@pytest.mark.parametrize("tune", ["size", "rd"])
@pytest.mark.parametrize("shape", [(72, 60), (24, 20, 28), (12, 10, 8, 6)])
def test_tune_choice_matches_oracle_sweep(tune, shape):
    """The encoder's tune sweep (latec/codec.py:171-262) against the oracle's
    restatement of it: in the reference-readable (compat) mode, where every
    candidate's stream bytes are the reference's, the same candidates are
    tried, the same (eb ratio, center, end mode) wins and the chosen stream is
    byte-identical."""
    from latec_b200 import fields

    x = fields.turbulence_jumps(shape, seed=11)
    eb = 2e-3
    lv, stride = (3, 8)
    lb = _lb()
    stream, st = lb.compress(x, eb, lb.InterpPredictor("cubic", lv, stride, 1), levels=lv,
                             anchor_stride=stride, tune=tune, entropy="compat")
    ostream, _, choice, n_cand = ocodec.tune_sweep(x, eb, tune, "cubic", lv, stride)
    assert st["tune_candidates"] == n_cand
    assert (st["eb_ratio"], st["interp_center"], st["interp_end_mode"]) == choice
    assert stream == ostream


def test_corrupted_streams_raise_not_hang():
    from latec_b200 import fields

    x = fields.grf_se((96, 80), 6.0, seed=4)
    lb = _lb()
    stream, _ = lb.compress(x, 1e-3, lb.InterpPredictor("cubic", 3, 8, 1), levels=3, anchor_stride=8)
    with pytest.raises(ValueError):
        lb.decompress(b"NOTLATEC" + stream[8:])
    with pytest.raises(ValueError):
        lb.decompress(stream[: len(stream) // 2])
    rs = np.random.RandomState(0)
    for _ in range(20):
        bad = bytearray(stream)
        pos = rs.randint(100, len(bad))
        bad[pos] ^= 1 << rs.randint(0, 8)
        try:
            out = lb.decompress(bytes(bad))
            assert out.shape == x.shape
        except (ValueError, KeyError, NotImplementedError):
            pass


def test_empty_stages_and_tiny_grids():
    lb = _lb()
    for shape, lv, stride in [((1, 1), 1, 2), ((1, 3), 2, 4), ((2, 1, 1), 3, 8), ((5, 5), 5, 16)]:
        x = np.random.RandomState(1).rand(*shape).astype(np.float32)
        if len(shape) == 3 and shape[-1] in (1, 3):
            continue
        stream, st = lb.compress(x, 1e-3, lb.InterpPredictor("cubic", lv, stride, 1), levels=lv,
                                 anchor_stride=stride)
        ostream, _ = ocodec.compress(x, 1e-3, levels_=lv, anchor_stride=stride, mode="native")
        assert stream == ostream
        assert np.abs(lb.decompress(stream) - x).max() <= 1e-3


def test_device_stream_roundtrip_equals_host_stream():
    """stream_out="device" keeps the container in HBM: same bytes as the host
    stream, decodable from the tensor without host copies of the payload."""
    import torch

    from latec_b200 import fields

    x = fields.turbulence_jumps((70, 64, 50), seed=12)
    lb = _lb()
    s_host, st = lb.compress(x, 1e-3, lb.InterpPredictor("cubic", 4, 16, 1), levels=4,
                             anchor_stride=16)
    xd = torch.from_numpy(x).cuda()
    s_dev, st2 = lb.compress(xd, 1e-3, lb.InterpPredictor("cubic", 4, 16, 1), levels=4,
                             anchor_stride=16, stream_out="device")
    assert s_dev.is_cuda and bytes(s_dev.cpu().numpy()) == s_host
    back = lb.decompress(s_dev, out="device")
    assert torch.equal(back, st2["recon"])
    assert np.array_equal(lb.decompress(s_host), st["recon"])


class _HostCubic:
    """A caller's predictor, the reference's duck-typed plugin
    (``predict(recon, known, pos)``): the oracle's cubic interpolation on the
    host, finding its stage by the mask it is given."""

    def __init__(self, shape, levels, stride):
        from oracle import interp, levels as olevels

        self.interp = interp
        self.plan = list(olevels.iter_plan(shape, levels, stride, 1))
        self.calls = 0

    def predict(self, recon, known, pos):
        self.calls += 1
        for mask, s, axes in self.plan:
            if np.array_equal(mask, pos):
                assert not np.any(known & pos)
                return self.interp.predict(recon, s, axes, np.flatnonzero(pos), "cubic", 0, 1)
        raise AssertionError("the predictor was given an unknown stage")


@pytest.mark.parametrize("shape,entropy", [((40, 36), "native"), ((17, 20, 11), "native"),
                                           ((40, 36), "compat")])
def test_caller_predictor_drives_the_closed_loop(shape, entropy):
    """Any predictor with ``predict(recon, known, pos)`` runs the codec, as in
    the reference: a host restatement of the cubic interpolation codes the
    payload InterpPredictor's fused kernels code, and decompress with its
    factory returns the same field."""
    from latec_b200 import fields
    from latec_b200.bitstream import Header

    lb = _lb()
    x = fields.grf_se(shape, 6.0, seed=4)
    lv, st = 2, 4
    host = _HostCubic(shape, lv, st)
    s_host, st_host = lb.compress(x, 1e-3, host, levels=lv, anchor_stride=st, eb_ratio=0.9,
                                  entropy=entropy)
    s_ref, st_ref = lb.compress(x, 1e-3, lb.InterpPredictor("cubic", lv, st, 1), levels=lv,
                                anchor_stride=st, eb_ratio=0.9, entropy=entropy)
    assert host.calls > 0
    hs = Header.unpack(bytes(s_host[:4096])).size
    assert Header.unpack(bytes(s_ref[:4096])).size == hs
    assert s_host[hs:] == s_ref[hs:]  # the same frame and stage records
    assert np.array_equal(st_host["recon"], st_ref["recon"])
    y = lb.decompress(s_host, predictor_factory=lambda h: _HostCubic(shape, lv, st))
    assert np.array_equal(y, st_ref["recon"])
    assert np.abs(y.astype(np.float64) - x).max() <= 1e-3
    with pytest.raises(ValueError):
        lb.decompress(s_host)  # the stream names no built-in predictor
