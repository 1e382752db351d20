"""Synthetic training fields for the learned predictor, in [0, 1]
(``sample_synthetic_batch``, ``latec/synthetic_data.py:176-332``, restated
with its helpers ``_gaussian_smooth`` :56-72, ``_warp`` :75-109,
``_turbulent_advect`` :112-145 and ``_add_discontinuities`` :148-174).

Per field, drawn from the numpy generator in the reference's order so a
seeded run gives the reference's fields:

* knobs: a base correlation length log-uniform in [min/2, max] of
  ``correlation``, jittered per axis by a random spread (isotropic to
  strongly anisotropic); a marginal warp (identity, signed power, tanh); the
  turbulent flag (probability ``turbulence_frac``) and its spectrum exponent
  p ~ U(0.7, 1.6); the number of hyperplane jumps (1..``max_discontinuities``
  with probability ``discontinuity_frac``);
* structure: white noise filtered through a mirror-doubled FFT (an exact
  reflecting boundary): a Gaussian of the per-axis lengths for smooth fields,
  |k|^-p with the mean removed for turbulent ones, plus half of a second
  realisation at twice the lengths;
* turbulent fields are advected through a smooth random flow: three
  backward multilinear warps along a frozen displacement of amplitude
  U(0.04, 0.10) x the shortest axis;
* the marginal warp on the standardised field, the jumps (random unit
  normal, threshold at a random interior quantile, height +-U(0.4, 1.5)
  standard deviations), and the robust scaling that maps the 1 % / 99 %
  quantiles to 0 / 1 with clipping.

The generation is plain PyTorch on ``device`` (FFT products and gathers): it
makes training data and is not part of the codec's path.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = ["sample_synthetic_batch", "warp_fields", "smooth_fields", "DEFAULTS"]

# the reference's distribution file (synthetic_dist.yaml): 4-D fields use
# correlation_4d, 2-D crops correlation_2d
DEFAULTS = {"turbulence_frac": 0.4, "max_discontinuities": 3, "discontinuity_frac": 0.25,
            "correlation_4d": (1.0, 8.0), "correlation_2d": (2.0, 32.0)}


@dataclass
class _Knobs:
    sigmas: list
    warp: int  # 0 identity, 1 signed power, 2 tanh
    warp_param: float
    turbulent: bool
    exponent: float
    cuts: int


def _draw_knobs(rng, ndim, correlation, turbulence_frac, max_disc, disc_frac):
    lo = min(correlation) * 0.5
    hi = max(correlation)
    base = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    spread = float(rng.uniform(0.0, 1.0))
    sigmas = [max(0.3, base * float(np.exp(rng.normal(0.0, spread)))) for _ in range(ndim)]
    warp = int(rng.integers(3))
    warp_param = float(rng.uniform(0.4, 3.0)) if warp == 1 else float(rng.uniform(1.5, 4.0))
    turbulent = bool(rng.random() < turbulence_frac)
    exponent = float(rng.uniform(0.7, 1.6))
    cuts = 0
    if max_disc > 0 and rng.random() < disc_frac:
        cuts = int(rng.integers(1, int(max_disc) + 1))
    return _Knobs(sigmas, warp, warp_param, turbulent, exponent, cuts)


def _freqs(shape, device):
    """Per axis: the frequencies of the mirror-doubled axis on the rfftn grid,
    shaped to broadcast along that axis."""
    import torch

    nd = len(shape)
    out = []
    for k, n in enumerate(shape):
        f = (torch.fft.rfftfreq if k == nd - 1 else torch.fft.fftfreq)(2 * n, device=device)
        out.append(f.reshape(tuple(len(f) if a == k else 1 for a in range(nd))))
    return out


def _mirror_filter(x, shape, apply):
    """Filter rows ``x`` (R, *shape) through the FFT of their even extension
    (each axis doubled by its mirror image: an exact reflecting boundary):
    ``apply(spectrum)`` returns the filtered spectrum."""
    import torch

    dims = tuple(range(1, len(shape) + 1))
    for ax in dims:
        x = torch.cat([x, x.flip(ax)], dim=ax)
    y = torch.fft.irfftn(apply(torch.fft.rfftn(x, dim=dims)), s=x.shape[1:], dim=dims)
    return y[(slice(None),) + tuple(slice(n) for n in shape)]


def smooth_fields(x, sigma, shape, device):
    """Isotropic Gaussian blur of rows ``x`` (R, *shape) with length ``sigma``
    (``_gaussian_smooth``)."""
    import torch

    def apply(spec):
        for f in _freqs(shape, device):
            g = torch.exp(-2.0 * (math.pi * f) ** 2 * sigma ** 2)
            spec = spec * g.reshape(1, *g.shape)
        return spec

    return _mirror_filter(x, shape, apply)


def warp_fields(field, disp, shape, device):
    """Sample rows ``field`` (B, *shape) at grid + ``disp`` ((B, ndim, *shape),
    cell units) by multilinear interpolation over the 2^ndim cell corners,
    reflecting coordinates at the boundary (``_warp``)."""
    import torch

    B, nd = field.shape[0], len(shape)
    strides = [int(np.prod(shape[k + 1:])) for k in range(nd)]
    grid = torch.stack(torch.meshgrid(*[torch.arange(n, device=device, dtype=torch.float32)
                                        for n in shape], indexing="ij"))
    pos = grid[None] + disp
    cell = torch.floor(pos)
    t = pos - cell
    cell = cell.long()
    flat = field.reshape(B, -1)
    out = torch.zeros_like(field)
    for corner in range(1 << nd):
        weight = torch.ones_like(field)
        idx = torch.zeros(field.shape, dtype=torch.long, device=device)
        for k in range(nd):
            up = (corner >> k) & 1
            n = shape[k]
            c = torch.remainder(cell[:, k] + up, 2 * n)
            c = torch.where(c >= n, 2 * n - 1 - c, c)
            weight = weight * (t[:, k] if up else 1.0 - t[:, k])
            idx = idx + c * strides[k]
        out = out + weight * torch.gather(flat, 1, idx.reshape(B, -1)).reshape(field.shape)
    return out


def _advect(field, knobs, rng, shape, device, iters=3):
    """Three warps of the turbulent rows along one smooth random flow each;
    the other rows get zero displacement (``_turbulent_advect``)."""
    import torch

    B, nd, shortest = field.shape[0], len(shape), min(shape)
    amp = np.array([float(rng.uniform(0.04, 0.10)) * shortest if k.turbulent else 0.0
                    for k in knobs], dtype=np.float32)
    if not amp.any():
        return field
    sigma = float(rng.uniform(0.18, 0.40) * shortest)
    white = torch.from_numpy(rng.standard_normal((B * nd, *shape)).astype(np.float32)).to(device)
    flow = smooth_fields(white, sigma, shape, device).reshape(B, nd, *shape)
    unit = [1] * nd
    std = flow.reshape(B, nd, -1).std(dim=2).clamp_min(1e-6)
    disp = flow / std.reshape(B, nd, *unit)
    disp = disp * torch.from_numpy(amp).to(device).reshape(B, 1, *unit)
    for _ in range(iters):
        field = warp_fields(field, disp, shape, device)
    return field


def _base_fields(knobs, rng, shape, device):
    """Fine realisation + half of an independent one at twice the lengths,
    rows filtered together: Gaussian (smooth rows) or |k|^-p (turbulent)."""
    import torch

    B, nd = len(knobs), len(shape)
    sig = torch.tensor([k.sigmas for k in knobs] + [[2.0 * s for s in k.sigmas] for k in knobs],
                       dtype=torch.float32, device=device)
    turb = torch.tensor([k.turbulent for k in knobs] * 2, dtype=torch.bool, device=device)
    p = torch.tensor([k.exponent for k in knobs] * 2, dtype=torch.float32, device=device)
    noise = torch.from_numpy(rng.standard_normal((2 * B, *shape)).astype(np.float32)).to(device)
    rows = (-1,) + (1,) * nd

    def apply(spec):
        gexp = torch.zeros((2 * B,) + spec.shape[1:], device=device)
        k2 = torch.zeros(spec.shape[1:], device=device)
        for a, f in enumerate(_freqs(shape, device)):
            f2 = f ** 2
            gexp = gexp + f2[None] * sig[:, a].reshape(rows) ** 2
            k2 = k2 + f2
        gauss = torch.exp(-2.0 * math.pi ** 2 * gexp)
        power = (k2[None] + 1e-8) ** (-0.5 * p.reshape(rows))
        power = torch.where(k2[None] > 0, power, torch.zeros_like(power))
        return spec * torch.where(turb.reshape(rows), power, gauss)

    x = _mirror_filter(noise, shape, apply)
    return x[:B] + 0.5 * x[B:]


def _finish(fi, knobs, rng, coords, shape, device):
    """Marginal warp, hyperplane jumps and robust [0, 1] scaling of one field."""
    import torch

    s = float(fi.std())
    if s >= 1e-8:
        z = (fi - fi.mean()) / s
        if knobs.warp == 1:
            z = z.sign() * z.abs() ** knobs.warp_param
        elif knobs.warp == 2:
            z = torch.tanh(knobs.warp_param * z)
        fi = z
    if knobs.cuts > 0:
        height = float(fi.std()) or 1.0
        nd = len(coords)
        for _ in range(knobs.cuts):
            normal = rng.standard_normal(nd)
            normal = normal / (np.linalg.norm(normal) + 1e-12)
            proj = sum(float(normal[k]) * coords[k] for k in range(nd))
            at = torch.quantile(proj.reshape(-1), float(rng.uniform(0.25, 0.75)))
            jump = float(rng.choice((-1.0, 1.0))) * float(rng.uniform(0.4, 1.5)) * height
            fi = fi + jump * (proj > at).to(fi.dtype)
    lo, hi = torch.quantile(fi.reshape(-1), torch.tensor([0.01, 0.99], device=device))
    if float(hi) <= float(lo):
        return torch.full(shape, 0.5, device=device)
    return ((fi - lo) / (hi - lo)).clamp(0.0, 1.0)


def sample_synthetic_batch(batch, shape, correlation, rng=None, randomize=True, device="cpu",
                           turbulence_frac=0.5, max_discontinuities=3, discontinuity_frac=1.0):
    """(batch, prod(shape)) float32 fields in [0, 1] on ``device``
    (``latec/synthetic_data.py:176-332``). ``randomize=False`` gives the
    deterministic smooth path: the exact ``correlation`` per axis, no warp,
    turbulence or jumps."""
    import torch

    shape = tuple(int(n) for n in shape)
    correlation = tuple(float(s) for s in correlation)
    rng = np.random.default_rng() if rng is None else rng
    nd = len(shape)
    if randomize:
        knobs = [_draw_knobs(rng, nd, correlation, turbulence_frac, max_discontinuities,
                             discontinuity_frac) for _ in range(int(batch))]
    else:
        knobs = [_Knobs(list(correlation), 0, 0.0, False, 1.0, 0) for _ in range(int(batch))]
    field = _base_fields(knobs, rng, shape, device)
    if randomize:
        field = _advect(field, knobs, rng, shape, device)
    coords = [torch.linspace(0.0, 1.0, n, device=device).reshape(
        tuple(n if a == k else 1 for a in range(nd))) for k, n in enumerate(shape)]
    out = [_finish(field[i], knobs[i], rng, coords, shape, device) for i in range(int(batch))]
    return torch.stack(out).reshape(int(batch), -1)
