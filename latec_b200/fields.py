"""Seeded synthetic fields with the shapes and statistics of the benchmark workloads.

The reference evaluates on scientific fields (SDRBench-style s3d, Kodak images,
The Well) that are not available offline; these generators stand in for them
with documented, seeded statistics:

* ``grf_se`` -- Gaussian random field with squared-exponential covariance
  ``C(r) = exp(-r^2 / (2 l^2))``: white noise filtered by ``sqrt(PSD)`` in
  Fourier space, standardised to mean 0 / variance 1 in float64.
* ``turbulence_jumps`` -- white noise shaped by ``|k|^(-(d/2 + 5/6))`` (so the
  shell-summed energy spectrum goes as ``k^-5/3`` in any rank), DC removed,
  unit variance, plus ``n_jumps`` random hyperplanes each adding a step of
  ``jump`` on one side, the plane offset at a random interior quantile.
* ``grf_aniso`` -- SE-covariance field with one correlation length per axis.
* ``mixed_4d`` -- element-wise average (weight 0.5 each) of an anisotropic
  GRF and a turbulence+jumps field, each normalised to unit variance first.

Everything is plain NumPy (``numpy.fft``), float64 internally, so a given seed
gives the same array on every machine with the same NumPy. ``device="cuda"``
runs the FFTs through torch on the GPU instead, for the large benchmark
fields; that array is seeded the same way but is not bitwise identical to the
NumPy one.
"""

from __future__ import annotations

import numpy as np


def _kgrid(shape):
    """Per-axis frequency vectors (cycles/sample) for an rfftn layout."""
    ks = [np.fft.fftfreq(n) for n in shape[:-1]]
    ks.append(np.fft.rfftfreq(shape[-1]))
    return ks


def _k2(shape, scales=None):
    """|k|^2 (optionally with per-axis scale factors) on the rfftn grid."""
    ks = _kgrid(shape)
    out = None
    for j, k in enumerate(ks):
        sh = [1] * len(shape)
        sh[j] = len(k)
        term = (k * (1.0 if scales is None else scales[j])) ** 2
        term = term.reshape(sh)
        out = term if out is None else out + term
    return out


def _filter_noise(shape, amp_fn, rng, device=None):
    noise = rng.standard_normal(shape)
    if device is not None and str(device).startswith("cuda"):
        import torch

        t = torch.as_tensor(noise, device=device)
        spec = torch.fft.rfftn(t)
        amp = torch.as_tensor(amp_fn(), device=device)
        out = torch.fft.irfftn(spec * amp, s=shape)
        return out
    spec = np.fft.rfftn(noise)
    spec *= amp_fn()
    return np.fft.irfftn(spec, s=shape, axes=tuple(range(len(shape))))


def _standardise(a):
    if hasattr(a, "cpu"):
        a = a - a.mean()
        return a / a.std()
    a = a - a.mean()
    sd = a.std()
    return a / sd if sd > 0 else a


def grf_se(shape, corr_len=16.0, seed=0, device=None):
    """SE-covariance Gaussian random field, unit variance, float32."""
    shape = tuple(int(n) for n in shape)
    rng = np.random.default_rng(seed)
    # PSD of exp(-r^2/(2 l^2)) is proportional to exp(-2 pi^2 l^2 |k|^2);
    # the filter is its square root.
    amp = lambda: np.exp(-(np.pi**2) * corr_len**2 * _k2(shape))  # noqa: E731
    f = _standardise(_filter_noise(shape, amp, rng, device))
    return _to_f32(f)


def grf_aniso(shape, corr_lens, seed=0, device=None):
    """SE-covariance field with one correlation length per axis."""
    shape = tuple(int(n) for n in shape)
    rng = np.random.default_rng(seed)
    amp = lambda: np.exp(-(np.pi**2) * _k2(shape, corr_lens))  # noqa: E731
    return _to_f32(_standardise(_filter_noise(shape, amp, rng, device)))


def turbulence_jumps(shape, seed=0, n_jumps=3, jump=1.0, device=None):
    """Power-law (Kolmogorov) turbulence plus random hyperplane steps."""
    shape = tuple(int(n) for n in shape)
    d = len(shape)
    rng = np.random.default_rng(seed)

    def amp():
        k2 = _k2(shape)
        with np.errstate(divide="ignore"):
            a = np.where(k2 > 0, k2 ** (-(d / 2.0 + 5.0 / 6.0) / 2.0), 0.0)
        return a

    f = _standardise(_filter_noise(shape, amp, rng, device))
    for _ in range(n_jumps):
        normal = rng.standard_normal(d)
        normal /= np.linalg.norm(normal)
        q = rng.uniform(0.2, 0.8)
        f = _add_plane(f, shape, normal, q, jump)
    return _to_f32(f)


def _add_plane(f, shape, normal, quantile, jump):
    # offset = the requested quantile of n.x over the grid, taken in closed
    # form from the projected coordinate range (uniform grid).
    lo = sum(min(0.0, c * (n - 1)) for c, n in zip(normal, shape))
    hi = sum(max(0.0, c * (n - 1)) for c, n in zip(normal, shape))
    off = lo + quantile * (hi - lo)
    if hasattr(f, "cpu"):
        import torch

        proj = None
        for j, (c, n) in enumerate(zip(normal, shape)):
            sh = [1] * len(shape)
            sh[j] = n
            t = (torch.arange(n, device=f.device, dtype=f.dtype) * float(c)).reshape(sh)
            proj = t if proj is None else proj + t
        return f + jump * (proj > off).to(f.dtype)
    proj = None
    for j, (c, n) in enumerate(zip(normal, shape)):
        sh = [1] * len(shape)
        sh[j] = n
        t = (np.arange(n, dtype=np.float64) * c).reshape(sh)
        proj = t if proj is None else proj + t
    return f + jump * (proj > off)


def mixed_4d(shape, seed=0, device=None):
    """0.5 * anisotropic GRF (per-axis l ~ U(1, 8)) + 0.5 * turbulence+jumps."""
    rng = np.random.default_rng(seed)
    lens = rng.uniform(1.0, 8.0, len(shape))
    a = grf_aniso(shape, lens, seed=seed + 1, device=device)
    b = turbulence_jumps(shape, seed=seed + 2, device=device)
    if hasattr(a, "cpu"):
        a, b = a.double(), b.double()
        return _to_f32(0.5 * _standardise(a) + 0.5 * _standardise(b))
    a, b = a.astype(np.float64), b.astype(np.float64)
    return _to_f32(0.5 * _standardise(a) + 0.5 * _standardise(b))


def _to_f32(f):
    if hasattr(f, "cpu"):
        import torch

        return f.to(torch.float32).contiguous()
    return np.ascontiguousarray(f, dtype=np.float32)
