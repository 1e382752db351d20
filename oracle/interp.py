"""Oracle restatement of the interpolation predictor (reference ``latec/predictor.py``).

Test infrastructure only (see ``oracle/__init__.py``).

``predict(recon, s, axes, flat, order, center, end_mode)`` evaluates the
per-point rule at the flat grid indices ``flat`` (the stage's points in
C order): for every candidate axis, the 1-D line interpolation from the taps at
``+-s`` and ``+-3s`` (``latec/predictor.py:97-156``), then the centre combine
over the point's own odd axes (``latec/predictor.py:286-314``). Arithmetic is
float64 on the gathered values in the reference's evaluation order; the result
is cast to float32 for a float32 reconstruction (``latec/predictor.py:315``)
and kept in float64 for the float64 path.
"""

from __future__ import annotations

import numpy as np

END_QUAD = 1
END_EXTRAP = 2


def _axis_interp(W, flat, coords, shape, gstrides, axis, s, order, end_mode):
    """One axis of ``latec/predictor.py:75-156`` (gather + line rule)."""
    ca = coords[axis]
    n = shape[axis]

    def gather(off):
        t = ca + off
        valid = (t >= 0) & (t < n)
        t = np.clip(t, 0, n - 1)
        return W[:, flat + (t - ca) * gstrides[axis]].astype(np.float64), valid

    Lm1, vm1 = gather(-s)
    Lp1, vp1 = gather(+s)
    lin = 0.5 * (Lm1 + Lp1)
    pred = lin
    Lm3, vm3 = gather(-3 * s)
    Lp3, vp3 = gather(+3 * s)
    if order == "cubic":
        cub = (-Lm3 + 9 * Lm1 + 9 * Lp1 - Lp3) / 16.0
        one_far = lin
        if end_mode & END_QUAD:
            one_far = np.where((vp3 & ~vm3)[None], (3 * Lm1 + 6 * Lp1 - Lp3) / 8.0,
                               np.where((vm3 & ~vp3)[None], (-Lm3 + 6 * Lm1 + 3 * Lp1) / 8.0, lin))
        pred = np.where((vm3 & vp3)[None], cub, one_far)
    both = vm1 & vp1
    left, right = Lm1, Lp1
    if end_mode & END_EXTRAP:
        left = np.where(vm3[None], 1.5 * Lm1 - 0.5 * Lm3, Lm1)
        right = np.where(vp3[None], 1.5 * Lp1 - 0.5 * Lp3, Lp1)
    return np.where(both[None], pred, np.where((vm1 & ~vp1)[None], left, right))


def predict(recon, s, axes, flat, order="cubic", center=0, end_mode=1):
    """Predictions ``(C, len(flat))`` for the stage points at flat indices ``flat``.

    ``recon`` is ``(C, *S)``; ``axes`` the stage's candidate axes (one axis for a
    weight-1 sub-stage, all axes for a fused one). ``latec/predictor.py:255-317``.
    """
    shape = recon.shape[1:]
    W = recon.reshape(recon.shape[0], -1)
    gstrides = np.cumprod((1,) + shape[:0:-1])[::-1].astype(np.int64)
    flat = np.asarray(flat, np.int64)
    coords = np.unravel_index(flat, shape)

    def odd(a):
        return (coords[a] & s) != 0

    def vpred(a):
        return _axis_interp(W, flat, coords, shape, gstrides, a, s, order, end_mode)

    if center == 0 or len(axes) == 1:
        total = count = None
        for a in axes:
            v = vpred(a)
            m = odd(a)[None].astype(np.float64)
            total = v * m if total is None else total + v * m
            count = m if count is None else count + m
        with np.errstate(invalid="ignore", divide="ignore"):
            out = total / count
    else:
        out = None
        for a in (reversed(axes) if center == 1 else axes):
            v = vpred(a)
            out = v if out is None else np.where(odd(a)[None], v, out)
    if recon.dtype == np.float64:
        return out
    return out.astype(np.float32)
