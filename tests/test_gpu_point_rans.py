"""Per-point rANS on the device (``latec/rans.py:270-301,332-357,546-616``)
against the CPU oracle, bit for bit, and against the reference's golden scale
levels."""

import numpy as np
import pytest

from oracle import point as opoint
from oracle import rans_model as orm
from tests.golden_io import load_npz

pytestmark = pytest.mark.gpu

RADIUS = 1 << 15


def _case(n, seed, peak=40):
    """Codes whose spread follows their level (like a scale head's output),
    with ~1 % outliers (code 0)."""
    rs = np.random.RandomState(seed)
    levels = rs.randint(0, 64, n).astype(np.uint8)
    scale = np.exp(np.log(1 / 16) + levels / 63.0 * np.log(4096 * 16)) / 8.0
    q = np.clip(np.rint(rs.laplace(0, scale)), -peak, peak).astype(np.int64)
    codes = (q + RADIUS).astype(np.uint32)
    codes[rs.rand(n) < 0.01] = 0
    return codes, levels


def test_scale_levels_match_golden():
    from latec_b200 import rans

    z = load_npz("rans.npz")
    got = rans.scale_to_level(z["scales"], 0.01)
    assert np.array_equal(got, z["scale_levels"])


@pytest.mark.parametrize("eb", [1e-6, 1e-3, 0.25])
def test_scale_levels_match_oracle_at_every_boundary(eb):
    import torch

    from latec_b200 import rans

    th = rans.level_thresholds(eb)
    around = np.concatenate([np.nextafter(th, np.float32(-np.inf)), th,
                             np.nextafter(th, np.float32(np.inf))]).astype(np.float32)
    rs = np.random.default_rng(12)
    rnd = np.exp(rs.uniform(np.log(eb / 32), np.log(eb * 8192), 20_000)).astype(np.float32)
    vals = np.concatenate([around, rnd, np.float32([0.0, 1e-30, 1e30, np.inf])])
    want = orm.scale_to_level(vals, eb)
    assert np.array_equal(rans.scale_to_level(vals, eb), want)
    # a CUDA tensor stays on the device
    t = rans.scale_to_level(torch.from_numpy(vals).cuda(), eb)
    assert t.is_cuda and np.array_equal(t.cpu().numpy(), want)


@pytest.mark.parametrize("mode", ["compat", "native"])
@pytest.mark.parametrize("n,kexp,shape", [(1, None, 0), (1000, 6, 0), (100_003, 6, 5),
                                          (70_000, None, 0)])
def test_point_rans_bytes_match_oracle(mode, n, kexp, shape):
    from latec_b200 import rans

    codes, levels = _case(n, seed=n)
    tables = rans.build_laplace_tables(1e-3, RADIUS)
    blob = rans.rans_encode(codes, levels, tables, kexp=kexp, shape=shape, mode=mode)
    want = opoint.rans_encode(codes, levels, RADIUS, kexp=kexp, shape=shape, mode=mode)
    assert blob == want
    back = rans.rans_decode(blob, levels, tables, kexp=kexp, shape=shape, mode=mode)
    assert back.dtype == np.uint32 and np.array_equal(back, codes)
    assert np.array_equal(opoint.rans_decode(blob, levels, RADIUS, kexp, shape, mode), codes)


def test_point_rans_levels_all_equal_and_sorted():
    from latec_b200 import rans

    tables = rans.build_laplace_tables(1e-3, RADIUS)
    for levels in (np.full(5000, 17, np.uint8), np.sort(np.random.RandomState(3).randint(0, 64, 5000)).astype(np.uint8)):
        codes, _ = _case(5000, 7)
        for mode in ("compat", "native"):
            blob = rans.rans_encode(codes, levels, tables, kexp=6, mode=mode)
            assert blob == opoint.rans_encode(codes, levels, RADIUS, kexp=6, mode=mode)
            assert np.array_equal(rans.rans_decode(blob, levels, tables, kexp=6, mode=mode), codes)


def test_point_model_bits_and_shape_match_oracle():
    from latec_b200 import rans

    codes, levels = _case(200_000, 5)
    tables = rans.build_laplace_tables(1e-3, RADIUS)
    for shape in (0, 3, 11):
        got = rans.model_bits(codes, levels, tables, kexp=6, shape=shape)
        want = orm.model_bits(codes, levels, RADIUS, 6, shape)
        assert got == pytest.approx(want, rel=1e-12)
    for sample in (0.05, 1.0):
        assert (rans.choose_shape(codes, levels, tables, 6, sample=sample)
                == orm.choose_shape(codes, levels, RADIUS, 6, sample=sample))


def test_point_rans_errors():
    from latec_b200 import rans

    tables = rans.build_laplace_tables(1e-3, RADIUS)
    codes, levels = _case(3000, 9)
    assert rans.rans_encode(np.zeros(0, np.uint32), np.zeros(0, np.uint8), tables) == b""
    assert rans.rans_decode(b"", np.zeros(0, np.uint8), tables).size == 0
    with pytest.raises(ValueError):
        rans.rans_decode(b"\0\0\0\0", np.zeros(0, np.uint8), tables)
    with pytest.raises(ValueError):
        rans.rans_encode(codes, levels[:-1], tables)
    with pytest.raises(ValueError):  # outside the kexp window
        rans.rans_encode(codes, levels, tables, kexp=3)
    with pytest.raises(ValueError):
        rans.rans_encode(codes, np.full(3000, 64, np.uint8), tables)
    for mode in ("compat", "native"):
        blob = rans.rans_encode(codes, levels, tables, kexp=6, mode=mode)
        with pytest.raises(ValueError):
            rans.rans_decode(blob[:-2], levels, tables, kexp=6, mode=mode)
        with pytest.raises(ValueError):
            rans.rans_decode(blob + b"\1\0\0\0", levels, tables, kexp=6, mode=mode)
