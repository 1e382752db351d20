"""Generate tests/golden/synthetic.npz from the reference's synthetic field
generator itself (``latec.synthetic_data.sample_synthetic_batch``), on the
CPU in float32, for seeded numpy generators (the package imports with the
test-only zstandard shim in ``_refshim``). The cases cover 2-D, 3-D and 4-D
shapes, smooth and turbulent (advected) rows, every marginal warp and the
hyperplane jumps, plus the deterministic ``randomize=False`` path.

    python tests/golden/make_synthetic_golden.py --ref PATH
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# name, batch, shape, correlation, seed, randomize, turbulence_frac,
# max_discontinuities, discontinuity_frac
CASES = [
    ("s2d", 6, (40, 36), (2.0, 32.0), 3, True, 0.5, 3, 1.0),
    ("s3d", 4, (12, 10, 14), (1.0, 8.0), 5, True, 0.5, 2, 0.5),
    ("s4d", 3, (6, 7, 5, 6), (1.0, 8.0), 8, True, 0.4, 3, 0.25),
    ("s2d_smooth_only", 3, (24, 30), (2.0, 16.0), 11, True, 0.0, 0, 1.0),
    ("s2d_fixed", 2, (20, 18), (3.0, 5.0), 2, False, 0.5, 3, 1.0),
]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference LATEC checkout")
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(HERE, "_refshim"))  # test-only zstandard shim
    sys.path.insert(0, args.ref)
    import torch
    from latec.synthetic_data import sample_synthetic_batch

    torch.manual_seed(0)
    out = {}
    for name, b, shape, corr, seed, rnd, tf, md, df in CASES:
        x = sample_synthetic_batch(b, shape, corr, np.random.default_rng(seed), randomize=rnd,
                                   device="cpu", turbulence_frac=tf, max_discontinuities=md,
                                   discontinuity_frac=df)
        out[name] = x.numpy().astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "synthetic.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
