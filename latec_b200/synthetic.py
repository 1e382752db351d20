"""Synthetic training fields for the learned predictor, in [0, 1]
(``latec/synthetic_data.py:176-332`` sample_synthetic_batch, restated).

Per field: with probability ``turbulence_frac`` a power-law spectrum
|k|^-p (p ~ U(1.5, 3.5), multi-scale turbulence), otherwise a squared-
exponential Gaussian random field with one correlation length per axis drawn
from ``correlation`` (default 1 to 8 samples); then up to
``max_discontinuities`` hyperplane steps of random orientation, position and
height; then the reference's robust scaling: the 1 % / 99 % quantiles map to
0 / 1 and the result is clipped. The reference additionally advects the
turbulent fields through a random flow; this generator does not.
"""

from __future__ import annotations

import numpy as np

from .fields import _add_plane, _k2

__all__ = ["sample_synthetic_batch"]


def _field(shape, rng, correlation, turbulence_frac, max_disc, device):
    import torch

    d = len(shape)
    noise = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(device)
    if rng.uniform() < turbulence_frac:
        p = rng.uniform(1.5, 3.5)
        k2 = _k2(shape)
        with np.errstate(divide="ignore"):
            amp = np.where(k2 > 0, k2 ** (-p / 2.0), 0.0)
    else:
        lens = rng.uniform(correlation[0], correlation[1], d)
        amp = np.exp(-(np.pi ** 2) * _k2(shape, lens))
    spec = torch.fft.rfftn(noise) * torch.from_numpy(amp.astype(np.float32)).to(device)
    f = torch.fft.irfftn(spec, s=shape)
    f = (f - f.mean()) / f.std().clamp_min(1e-12)
    for _ in range(int(rng.integers(0, max_disc + 1))):
        normal = rng.standard_normal(d)
        normal /= np.linalg.norm(normal)
        f = _add_plane(f, shape, normal, rng.uniform(0.2, 0.8), rng.uniform(-2.0, 2.0))
    q = torch.quantile(f.reshape(-1), torch.tensor([0.01, 0.99], device=device))
    lo, hi = float(q[0]), float(q[1])
    if hi <= lo:
        return torch.full(shape, 0.5, device=device)
    return ((f - lo) / (hi - lo)).clamp(0.0, 1.0)


def sample_synthetic_batch(batch, shape, rng=None, device="cuda", correlation=(1.0, 8.0),
                           turbulence_frac=0.5, max_discontinuities=3):
    """(batch, prod(shape)) float32 fields in [0, 1] on ``device``."""
    import torch

    rng = rng if rng is not None else np.random.default_rng(0)
    shape = tuple(int(n) for n in shape)
    fs = [_field(shape, rng, correlation, turbulence_frac, max_discontinuities, device)
          for _ in range(int(batch))]
    return torch.stack(fs).reshape(int(batch), -1).contiguous()
