"""Oracle restatement of the error-bounded quantizer (reference ``latec/quantizer.py``).

Test infrastructure only (see ``oracle/__init__.py``).

float32 path (``latec/quantizer.py:28-120``): ``q = rint((f64(x) - f64(p)) / f64(2 eb))``;
in range iff ``|q| < radius``; ``code = q + radius`` else 0; the candidate
reconstruction is ``f32(f64(p) + f64(2 eb) * (code - radius))`` and the point is
demoted to an outlier (code 0, exact value kept in scan order) unless
``|x - recon| <= f32(eb)`` in float32.

float64 path (new; the reference rejects float64 input): the same steps with
``x``, ``p`` and the reconstruction kept in float64 and the bound checked in
float64, ``|x - recon| <= eb``.
"""

from __future__ import annotations

import numpy as np


def quantize(x, pred, eb, radius=1 << 15, round_output=False):
    """Return ``(codes uint32, outliers)``; float32 or float64 by ``x.dtype``.

    ``round_output`` verifies against the rounded reconstruction, for integer
    sources (``latec/quantizer.py:71-73``)."""
    if eb <= 0:
        raise ValueError(f"error bound must be > 0, got {eb}")
    f64 = np.asarray(x).dtype == np.float64
    dt = np.float64 if f64 else np.float32
    x = np.asarray(x, dt).ravel()
    pred = np.asarray(pred, dt).ravel()
    w = np.float64(2.0 * eb)
    with np.errstate(invalid="ignore", over="ignore"):
        qf = np.rint((x.astype(np.float64) - pred.astype(np.float64)) / w)
        in_range = np.abs(qf) < radius
        q = np.where(in_range, qf, 0).astype(np.int64)
        codes = np.where(in_range, q + radius, 0).astype(np.uint32)
        recon = recon_from_codes(pred, codes, eb, radius)
        if round_output:
            recon = np.rint(recon)
        if f64:
            ok = in_range & (np.abs(x - recon) <= np.float64(eb))
        else:
            ok = in_range & (np.abs(x - recon) <= np.float32(eb))
    codes[~ok] = 0
    return codes, x[codes == 0].copy()


def recon_from_codes(pred, codes, eb, radius):
    """``latec/quantizer.py:114-120``; float64 path keeps float64."""
    q = codes.astype(np.int64) - radius
    r = np.asarray(pred).astype(np.float64) + np.float64(2.0 * eb) * q
    return r if np.asarray(pred).dtype == np.float64 else r.astype(np.float32)


def dequantize(pred, codes, outliers, eb, radius=1 << 15):
    """``latec/quantizer.py:90-111``."""
    pred = np.asarray(pred).ravel()
    codes = np.asarray(codes, np.uint32).ravel()
    recon = recon_from_codes(pred, codes, eb, radius)
    z = codes == 0
    if int(z.sum()) != len(outliers):
        raise ValueError("outlier count mismatch")
    recon[z] = outliers
    return recon
