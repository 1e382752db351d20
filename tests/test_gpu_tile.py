"""The fused levels (five sub-stages of a 3-D level in one launch, over column
tiles of the level's lattice staged in shared memory with a halo) give exactly
the per-stage launches' results: the same stream bytes, reconstruction and
decode. Mode 1 fuses the finest level, mode 3 every level whatever its size
(coarser levels run on their lattice), mode 2 (the default) every level of at
least 2^18 points."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # shape, levels, stride, dtype, center, end_mode, order, radius
    ((64, 64, 64), 3, 8, np.float32, 0, 1, "cubic", 1 << 15),
    ((65, 47, 33), 3, 8, np.float32, 0, 3, "cubic", 1 << 15),
    ((61, 40, 37), 2, 4, np.float32, 1, 0, "cubic", 1 << 15),
    ((37, 70, 131), 3, 8, np.float32, 2, 2, "cubic", 1 << 15),
    ((130, 40, 20), 3, 8, np.float32, 0, 1, "cubic", 1 << 15),
    ((48, 50, 44), 3, 8, np.float64, 0, 1, "cubic", 1 << 15),
    ((45, 37, 70), 3, 8, np.float64, 2, 3, "cubic", 1 << 15),
    ((70, 66, 30), 3, 8, np.float32, 0, 1, "linear", 1 << 15),
    ((33, 65, 66), 3, 8, np.float32, 0, 1, "cubic", 8),  # many outliers
    ((34, 20, 70), 2, 4, np.float64, 1, 1, "linear", 4),
    ((3, 5, 200), 2, 4, np.float32, 0, 1, "cubic", 1 << 15),
    ((2, 2, 2), 1, 2, np.float32, 0, 1, "cubic", 1 << 15),
]


DEFAULT_MODE = 0


def _mode(m):
    from latec_b200 import _lib

    _lib.check(_lib.load().latec_set_tile_mode(m))


@pytest.mark.parametrize("case", CASES,
                         ids=lambda c: "x".join(map(str, c[0])) + c[3].__name__ + c[6] + str(c[7]))
def test_tile_levels_match_per_stage_launches(case):
    import torch

    import latec_b200 as lb
    from latec_b200 import _lib, fields

    shape, lv, st, dt, center, em, order, radius = case
    x = fields.turbulence_jumps(shape, seed=sum(shape) + lv, device="cuda").to(
        torch.float64 if dt == np.float64 else torch.float32)
    mm = torch.aminmax(x)
    eb = 1e-4 * (float(mm.max.item()) - float(mm.min.item()))
    lib = _lib.load()
    try:
        outs, launches = [], []
        for mode in (0, 1, 3, 2):
            _mode(mode)
            pred = lb.InterpPredictor(order, lv, st, 1, center=center, end_mode=em)
            n0 = lib.latec_launch_count()
            s, stt = lb.compress(x, eb, pred, levels=lv, anchor_stride=st, radius=radius,
                                 recon="device")
            n1 = lib.latec_launch_count()
            d = lb.decompress(s, out="device")
            launches.append((n1 - n0, lib.latec_launch_count() - n1))
            outs.append((s, stt, d))
        s0, st0, d0 = outs[0]
        r0 = st0["recon"]
        assert torch.equal(d0, r0)
        for s, stt, d in outs[1:]:
            assert s == s0
            assert torch.equal(stt["recon"], r0)
            assert torch.equal(d, r0)
            assert stt["stage_outliers"] == st0["stage_outliers"]
            for key in ("stage_pred_sae", "stage_pred_sse", "stage_recon_sae", "stage_recon_sse",
                        "stage_recon_max"):
                np.testing.assert_allclose(stt[key], st0[key], rtol=1e-9, atol=0, err_msg=key)
        assert float((d0.double() - x.double()).abs().max().item()) <= eb
        if radius < 100:
            assert sum(st0["stage_outliers"]) > 100  # the outlier paths ran
        if min(shape) >= 4:  # a fused level replaced five stage launches each way
            assert launches[1][1] < launches[0][1]
    finally:
        _mode(DEFAULT_MODE)


def test_tile_mode_is_deterministic():
    import torch

    import latec_b200 as lb
    from latec_b200 import fields

    x = fields.turbulence_jumps((96, 80, 136), seed=5, device="cuda")
    mm = torch.aminmax(x)
    eb = 1e-4 * (float(mm.max.item()) - float(mm.min.item()))
    pred = lb.InterpPredictor("cubic", 4, 16, 1)
    try:
        _mode(1)
        a, sa = lb.compress(x, eb, pred, levels=4, anchor_stride=16, recon="device")
        b, sb = lb.compress(x, eb, pred, levels=4, anchor_stride=16, recon="device")
    finally:
        _mode(DEFAULT_MODE)
    assert a == b
    assert sa["stage_recon_sse"] == sb["stage_recon_sse"]
    assert sa["stage_pred_sae"] == sb["stage_pred_sae"]


def test_tile_mode_rejects_bad_values():
    from latec_b200 import _lib

    lib = _lib.load()
    assert lib.latec_set_tile_mode(4) != 0
    assert lib.latec_set_tile_mode(-1) != 0
    assert lib.latec_set_tile_mode(0) == 0
    assert lib.latec_set_tile_mode(DEFAULT_MODE) == 0
