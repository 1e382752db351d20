"""The level kernels (all sub-stages of a level in one launch, slab by slab,
with in-launch dependencies) give exactly the per-stage launches' results.
Mode 2 forces them on every level that qualifies, so small grids exercise
them too."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # shape, levels, stride, dtype, center, end_mode, order
    ((64, 64, 64), 3, 8, np.float32, 0, 1, "cubic"),
    ((65, 47, 33), 3, 8, np.float32, 0, 3, "cubic"),
    ((61, 40, 37), 2, 4, np.float32, 1, 0, "cubic"),
    ((300, 257), 4, 16, np.float32, 0, 1, "cubic"),
    ((20, 18, 16, 14), 2, 4, np.float32, 2, 2, "cubic"),
    ((48, 50, 44), 3, 8, np.float64, 0, 1, "cubic"),
    ((70, 66, 30), 3, 8, np.float32, 0, 1, "linear"),
]


def _mode(m):
    from latec_b200 import _lib

    _lib.check(_lib.load().latec_set_level_mode(m))


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])) + c[3].__name__)
def test_level_kernels_match_per_stage_launches(case):
    import torch

    import latec_b200 as lb
    from latec_b200 import fields

    shape, lv, st, dt, center, em, order = case
    x = fields.turbulence_jumps(shape, seed=len(shape) + lv, device="cuda").to(
        torch.float64 if dt == np.float64 else torch.float32)
    mm = torch.aminmax(x)
    eb = 1e-4 * (float(mm.max.item()) - float(mm.min.item()))
    try:
        from latec_b200 import _lib

        lib = _lib.load()
        _lib.check(lib.latec_set_tile_mode(0))  # per-stage launches on the finest level too
        outs, launches = [], []
        for mode in (0, 2):
            _mode(mode)
            pred = lb.InterpPredictor(order, lv, st, 1, center=center, end_mode=em)
            s, stt = lb.compress(x, eb, pred, levels=lv, anchor_stride=st, recon="device")
            n0 = lib.latec_launch_count()
            d = lb.decompress(s, out="device")
            launches.append(lib.latec_launch_count() - n0)
            outs.append((s, stt["recon"], d))
        (s0, r0, d0), (s2, r2, d2) = outs
        if len(shape) == 3 and dt == np.float32:
            assert launches[1] < launches[0]  # the level kernels did run
        assert launches[1] <= launches[0]
        assert s0 == s2
        assert torch.equal(d0, r0) and torch.equal(d2, r0) and torch.equal(r2, r0)
        assert float((d2.double() - x.double()).abs().max().item()) <= eb
    finally:
        _mode(0)
        from latec_b200 import _lib

        _lib.check(_lib.load().latec_set_tile_mode(0))  # the default
