"""The synthetic training-field generator (latec_b200.synthetic) against the
reference's own fields for the same seeds (tests/golden/synthetic.npz, made
by tests/golden/make_synthetic_golden.py), and properties of its warp."""

import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "synthetic.npz")

CASES = [
    ("s2d", 6, (40, 36), (2.0, 32.0), 3, True, 0.5, 3, 1.0),
    ("s3d", 4, (12, 10, 14), (1.0, 8.0), 5, True, 0.5, 2, 0.5),
    ("s4d", 3, (6, 7, 5, 6), (1.0, 8.0), 8, True, 0.4, 3, 0.25),
    ("s2d_smooth_only", 3, (24, 30), (2.0, 16.0), 11, True, 0.0, 0, 1.0),
    ("s2d_fixed", 2, (20, 18), (3.0, 5.0), 2, False, 0.5, 3, 1.0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_fields_match_the_reference_generator(case):
    from latec_b200.synthetic import sample_synthetic_batch

    name, b, shape, corr, seed, rnd, tf, md, df = case
    want = np.load(GOLDEN)[name]
    got = sample_synthetic_batch(b, shape, corr, np.random.default_rng(seed), randomize=rnd,
                                 device="cpu", turbulence_frac=tf, max_discontinuities=md,
                                 discontinuity_frac=df).numpy()
    assert got.shape == want.shape == (b, int(np.prod(shape)))
    assert got.min() >= 0.0 and got.max() <= 1.0
    # the same float32 operations in the same order on the CPU: the same bits
    np.testing.assert_array_equal(got, want)


def test_generator_draws_every_branch():
    """The fixture seeds exercise turbulent and smooth rows, all marginal
    warps and the jumps."""
    from latec_b200.synthetic import _draw_knobs

    kinds, turb, cuts = set(), set(), set()
    for name, b, shape, corr, seed, rnd, tf, md, df in CASES[:3]:
        rng = np.random.default_rng(seed)
        for _ in range(b):
            k = _draw_knobs(rng, len(shape), corr, tf, md, df)
            kinds.add(k.warp)
            turb.add(k.turbulent)
            cuts.add(k.cuts > 0)  # a batch's knobs are the generator's first draws
    assert kinds == {0, 1, 2} and turb == {True, False} and cuts == {True, False}


def test_warp_with_zero_displacement_is_the_identity():
    import torch

    from latec_b200.synthetic import warp_fields

    shape = (7, 9, 5)
    f = torch.rand((2, *shape))
    out = warp_fields(f, torch.zeros((2, 3, *shape)), shape, "cpu")
    assert torch.equal(out, f)


def test_warp_shifts_a_ramp_and_reflects_at_the_boundary():
    import torch

    from latec_b200.synthetic import warp_fields

    shape = (16, 12)
    ramp = torch.arange(16, dtype=torch.float32)[:, None].expand(shape).contiguous()[None]
    disp = torch.zeros((1, 2, *shape))
    disp[:, 0] = 2.25
    out = warp_fields(ramp, disp, shape, "cpu")[0]
    # interior: sampled 2.25 cells further along axis 0 (linear in the cell)
    assert torch.allclose(out[:13], ramp[0, :13] + 2.25, atol=1e-5)
    # past the end the coordinate reflects: position 15 + 2.25 = 17.25 mirrors
    # to 13.75 (between cells 14 and 13 of the reversed copy)
    assert torch.allclose(out[15], torch.full((12,), 13.75), atol=1e-5)
