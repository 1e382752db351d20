"""Laplace-mixture rANS model on the host (reference ``latec/rans.py``).

The tables are the reference's: per-level continuous Laplace bin weights over
the ``[eb/16, 4096 eb]`` scale grid, the 21-entry mixture dictionary, the
outlier-marker dictionary, and the largest-remainder 24-bit quantisation.
They are deterministic NumPy, built once per ``(kexp, shape, owx)`` and cached
on the host and, per row, on the device (encoder symbols with exact
reciprocal divisions, decoder buckets). The stage-constant model fit runs the
reference's float32 matrix-vector product on the stage histogram that the
quantizer kernel accumulated on the device.
"""

from __future__ import annotations

import math
from collections import OrderedDict
from functools import lru_cache

import numpy as np

SCALE_LO_DIV = 16.0
SCALE_HI_MULT = 4096.0
N_LEVELS = 64
PRECISION = 24
SHAPES = ((0, 0.0),) + tuple((d, w) for d in (4, 8, 16, 24) for w in (0.02, 0.05, 0.12, 0.25, 0.45))
OUTLIER_WEIGHTS = (0.0, 2.0**-13, 2.0**-10, 2.0**-8, 2.0**-6, 2.0**-4, 2.0**-2, 0.5)
WIDE_KEXP = 13
SEG = 1 << 22          # the reference accumulates its float32 histogram per 2^22 codes
HWIN = 256             # device histogram window (|q| < HWIN), see interp_kernels.cuh
LITERAL_MIN = 1 << 12
NBUCKET = 1 << 10      # decoder bucket table entries per CDF row (rans_kernels.cuh)
ENC_BYTES = 32          # encoder entry per symbol (EncSym in rans_kernels.cuh)
LITERAL_SCOUT_SLACK = 0.85

# Native lane coder chunking: keep the 64-bit final lane states under ~1/64 of
# a stage's modelled bits, with 16..8192 symbols per lane.
LANES_KMIN, LANES_KMAX, LANES_BITS_PER_WARP = 16, 8192, 131072


def full_kexp(radius):
    return max(1, int(int(radius) - 1).bit_length())


def shape_ids(kexp):
    """Dictionary entries the encoder considers (``latec/rans.py:194-201``)."""
    if kexp < WIDE_KEXP:
        return tuple(range(len(SHAPES)))
    return (0,) + tuple(i for i, (_d, w) in enumerate(SHAPES) if w == 0.02)


def _laplace_cdf(x, b):
    z = np.clip(x / b, -700.0, 700.0)
    return np.where(x < 0, 0.5 * np.exp(z), 1.0 - 0.5 * np.exp(-z))


@lru_cache(maxsize=32)
def level_weights(kexp, n_levels=N_LEVELS):
    """Row-normalised Laplace bin weights per scale level (``latec/rans.py:246-267``)."""
    span = (1 << kexp) - 1
    lo, hi = 1.0 / SCALE_LO_DIV, SCALE_HI_MULT
    grid = np.exp(np.linspace(np.log(lo), np.log(hi), n_levels)).astype(np.float64)
    q = np.arange(-span, span + 1, dtype=np.float64)
    left, right = q * 2.0 - 1.0, q * 2.0 + 1.0
    w = np.empty((n_levels, 2 * span + 2), np.float64)
    for i, b in enumerate(grid):
        w[i, 1:] = _laplace_cdf(right, b) - _laplace_cdf(left, b)
        w[i, 0] = w[i, 1:].max() * 1e-9
    w /= w.sum(1, keepdims=True)
    return w


@lru_cache(maxsize=512)
def shaped_weights(kexp, shape, n_levels=N_LEVELS):
    """Mixture entry ``shape``: (1-w) p[level] + w p[level+d] (``latec/rans.py:376-384``)."""
    weights = level_weights(kexp, n_levels)
    d, w = SHAPES[shape]
    if not w:
        return weights
    return (1.0 - w) * weights + w * weights[np.minimum(np.arange(n_levels) + d, n_levels - 1)]


def with_outlier_weight(weights, owx):
    """``latec/rans.py:172-180``."""
    ow = OUTLIER_WEIGHTS[int(owx)]
    if not ow:
        return weights
    out = weights.copy()
    out[:, 1:] *= (1.0 - ow) / out[:, 1:].sum(1, keepdims=True)
    out[:, 0] = ow
    return out


def quantize_pmf_rows(weights, total):
    """Counts >= 1 summing to ``total`` per row, largest remainders first
    (``latec/rans.py:676-722``)."""
    w = np.asarray(weights, np.float64)
    _, alphabet = w.shape
    scaled = w / w.sum(1, keepdims=True) * total
    floor = np.floor(scaled)
    pmf = np.maximum(floor.astype(np.int64), 1)
    frac = scaled - floor
    diff = total - pmf.sum(1)
    up = np.flatnonzero(diff > 0)
    if len(up):
        bulk, rem = np.divmod(diff[up], alphabet)
        pmf[up] += bulk[:, None]
        order = np.argsort(-frac[up], axis=1, kind="stable")
        rank = np.empty_like(order)
        np.put_along_axis(rank, order, np.broadcast_to(np.arange(alphabet), order.shape), axis=1)
        pmf[up] += rank < rem[:, None]
    down = np.flatnonzero(diff < 0)
    if len(down):
        need = -diff[down]
        order = np.argsort(frac[down], axis=1, kind="stable")
        avail = np.take_along_axis(pmf[down], order, axis=1) - 1
        cum = np.cumsum(avail, axis=1)
        take = np.clip(need[:, None] - (cum - avail), 0, avail)
        if np.any(take.sum(1) < need):
            raise ValueError("could not normalize PMF at requested precision")
        rows = pmf[down]
        np.put_along_axis(rows, order, np.take_along_axis(rows, order, axis=1) - take, axis=1)
        pmf[down] = rows
    return pmf.astype(np.uint32)


@lru_cache(maxsize=256)
def cdfs(kexp, shape=0, owx=0, n_levels=N_LEVELS, precision=PRECISION):
    """``(n_levels, alphabet + 1)`` uint32 CDF rows (``latec/rans.py:304-329``)."""
    alphabet = 2 * ((1 << kexp) - 1) + 2
    if alphabet > (1 << precision):
        raise ValueError("precision is too small for the quantizer alphabet")
    weights = with_outlier_weight(shaped_weights(kexp, shape, n_levels), owx)
    out = np.empty((n_levels, alphabet + 1), np.uint32)
    out[:, 0] = 0
    out[:, 1:] = np.cumsum(quantize_pmf_rows(weights, 1 << precision), axis=1, dtype=np.uint64)
    return out


@lru_cache(maxsize=512)
def neg_log2_weights(kexp, shape, owx, n_levels=N_LEVELS, precision=PRECISION):
    """``latec/rans.py:387-392``."""
    weights = with_outlier_weight(shaped_weights(kexp, shape, n_levels), owx)
    return -np.log2(np.maximum(weights, 1.0 / (1 << precision))).astype(np.float32)


_LOG_OW = np.log(np.maximum(np.asarray(OUTLIER_WEIGHTS, np.float64), 1e-12))


def choose_outlier_weight(n_outliers, n_codes):
    """``latec/rans.py:162-169``."""
    if n_codes <= 0 or n_outliers <= 0:
        return 0
    rate = n_outliers / n_codes
    return int(np.argmin(np.abs(_LOG_OW - np.log(rate))))


def choose_outlier_weights(n_outliers, n_codes):
    """Vector form of ``choose_outlier_weight`` (same float64 operations)."""
    n_out = np.asarray(n_outliers, np.float64)
    n = np.asarray(n_codes, np.float64)
    ok = (n > 0) & (n_out > 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        rate = np.where(ok, n_out / np.where(n > 0, n, 1.0), 1.0)
        idx = np.argmin(np.abs(_LOG_OW[None, :] - np.log(rate)[:, None]), axis=1)
    return np.where(ok, idx, 0).astype(np.int64)


def kexp_from_maxq(maxq):
    """``latec/rans.py:70-80`` from the device's max |q| over in-range codes."""
    return max(1, int(maxq).bit_length())


def stage_hist_f32(n_items, kexp, radius, seg_window, total_codes):
    """The reference's float32 stage histogram over the reduced alphabet.

    ``seg_window``: ``(n_segments, 2*HWIN)`` uint32 device counts per 2^22-code
    segment (bin 0 outliers, bin ``q + HWIN`` for ``|q| < HWIN``);
    ``total_codes``: per code value counts for ``|q| >= HWIN`` (65536 bins).
    The float32 accumulation of ``latec/rans.py:414-420`` (float32 += int64 per
    segment) is replayed exactly for every window bin; bins outside the window
    only have totals, which is exact unless one such bin exceeds 2^24 codes.
    """
    span = (1 << kexp) - 1
    alphabet = 2 * span + 2
    seg = np.asarray(seg_window, np.int64)
    acc = np.zeros(seg.shape[1], np.float32)
    if seg.shape[0] == 1:
        acc = seg[0].astype(np.float32)
    else:
        for row in seg:
            acc = (acc.astype(np.float64) + row).astype(np.float32)
    hist = np.zeros(alphabet, np.float32)
    hist[0] = acc[0]
    lo = max(-span, -(HWIN - 1))
    hi = min(span, HWIN - 1)
    # symbol for q is q + span + 1
    hist[lo + span + 1:hi + span + 2] = acc[lo + HWIN:hi + HWIN + 1]
    if span >= HWIN:
        codes = np.arange(-span, span + 1) + radius
        q = codes - radius
        outside = np.abs(q) >= HWIN
        hist[(q[outside] + span + 1)] = np.asarray(total_codes, np.int64)[codes[outside]].astype(np.float32)
    return hist


def fit_const_level(hist, n_codes, kexp):
    """(level, shape, owx, bits) minimising the stage cost (``latec/rans.py:395-430``)."""
    if n_codes == 0:
        return 0, 0, 0, 0.0
    owx = choose_outlier_weight(int(hist[0]), n_codes)
    best = (np.inf, 0, 0)
    for sid in shape_ids(int(kexp)):
        cost = neg_log2_weights(int(kexp), int(sid), owx) @ hist
        level = int(cost.argmin())
        if cost[level] < best[0]:
            best = (float(cost[level]), level, int(sid))
    return best[1], best[2], owx, best[0]


def lanes_K(n, model_bits):
    """Symbols per lane per chunk of the native coder for a stage."""
    lo = -(-n // (32 * LANES_KMAX))
    hi = -(-n // (32 * LANES_KMIN))
    warps = max(lo, min(hi, max(1, int(math.floor(model_bits / LANES_BITS_PER_WARP)))))
    return -(-n // (32 * warps))


def fast_quantize_rows(cdf_rows):
    """constriction's ``Categorical(probs, perfect=False)`` re-quantisation of
    integer CDF rows (float32 running sum scaled by (2^24 - n) / sum, one count
    of slack per symbol): the compatibility coder's wire model."""
    rows = np.asarray(cdf_rows)
    n = rows.shape[1] - 1
    probs = np.diff(rows.astype(np.int64), axis=1).astype(np.float32)
    norm = probs.sum(1, dtype=np.float32)  # exact: integer counts summing to 2^24
    scale = np.float32((1 << PRECISION) - n) / norm
    cum = np.concatenate([np.zeros((rows.shape[0], 1), np.float32),
                          np.cumsum(probs, axis=1, dtype=np.float32)[:, :-1]], axis=1)
    left = (cum * scale[:, None]).astype(np.uint32) + np.arange(n, dtype=np.uint32)
    out = np.empty_like(rows, dtype=np.uint32)
    out[:, :n] = left
    out[:, n] = 1 << PRECISION
    if np.any(np.diff(out.astype(np.int64), axis=1) <= 0):
        raise ValueError("compatibility model has an empty symbol")
    return out


def narrow(codes, radius, kexp):
    span = (1 << int(kexp)) - 1
    q = np.asarray(codes).astype(np.int64) - int(radius)
    return np.where(np.asarray(codes) == 0, 0, q + span + 1)


def widen(syms, radius, kexp):
    span = (1 << int(kexp)) - 1
    codes = np.asarray(syms).astype(np.int64) - span - 1 + int(radius)
    return np.where(np.asarray(syms) == 0, 0, codes).astype(np.uint32)


def literal_dtype(kexp):
    return np.dtype(np.uint8 if int(kexp) <= 7 else np.uint16)


def narrow_literals(codes, radius, kexp):
    """``narrow(codes, radius, kexp)`` in ``literal_dtype(kexp)``: the symbol
    bytes of a literal (zstd) stage. Works in 16-bit modular arithmetic: an
    in-range code c maps to c - radius + 2^kexp < 2^(kexp + 1) <= 2^16, and an
    outlier (code 0) to 0."""
    c = np.asarray(codes, np.uint16)
    s = c + np.uint16(((1 << int(kexp)) - int(radius)) % (1 << 16))
    s[c == 0] = 0
    return s.astype(literal_dtype(kexp), copy=False)


# ------------------------------------------------------------------ device tables

class DeviceTables:
    """Device copies of CDF rows with their encoder symbols and decoder
    buckets, keyed by ``(mode, kexp, shape, owx, level)`` (``level`` None =
    all 64 rows), evicted least-recently-used by bytes."""

    def __init__(self, budget_bytes=1 << 30):
        self.budget = budget_bytes
        self.used = 0
        self.cache: "OrderedDict[tuple, tuple]" = OrderedDict()

    def get(self, mode, kexp, shape, owx, level=None, device=None):
        import torch

        from . import _lib

        key = (mode, kexp, shape, owx, level, str(device))
        hit = self.cache.get(key)
        if hit is not None:
            self.cache.move_to_end(key)
            return hit
        rows = cdfs(kexp, shape, owx)
        if level is not None:
            rows = rows[level:level + 1]
        if mode == _lib.RANS_COMPAT:
            rows = fast_quantize_rows(rows)
        alphabet = rows.shape[1] - 1
        dev = torch.device(device) if device is not None else torch.device("cuda")
        cdf = torch.from_numpy(np.ascontiguousarray(rows)).to(dev)
        enc = torch.empty(rows.shape[0] * (alphabet + 1) * ENC_BYTES, dtype=torch.uint8, device=dev)
        bucket = torch.empty(rows.shape[0] * NBUCKET, dtype=torch.int16, device=dev)
        lib = _lib.load()
        _lib.check(lib.latec_rans_build_tables(cdf.data_ptr(), alphabet, rows.shape[0],
                                               enc.data_ptr(), bucket.data_ptr(),
                                               _lib.stream_ptr()), "latec_rans_build_tables")
        entry = (cdf, enc, bucket, alphabet)
        size = cdf.numel() * 4 + enc.numel() + bucket.numel() * 2
        self.cache[key] = entry
        self.used += size
        while len(self.cache) > 1 and self.used > self.budget:
            _, old = self.cache.popitem(last=False)
            self.used -= old[0].numel() * 4 + old[1].numel() + old[2].numel() * 2
        return entry


device_tables = DeviceTables()


class DeviceWeights:
    """Device copies of the stacked -log2 weight tables of every dictionary
    entry the encoder considers, ``(n_shapes, 64, alphabet)`` float32, keyed by
    ``(kexp, owx)`` (the native-mode fit's operand)."""

    def __init__(self, budget_bytes=1 << 30):
        self.budget, self.used = budget_bytes, 0
        self.cache: "OrderedDict[tuple, tuple]" = OrderedDict()

    def get(self, kexp, owx, device):
        import torch

        key = (kexp, owx, str(device))
        hit = self.cache.get(key)
        if hit is not None:
            self.cache.move_to_end(key)
            return hit
        ids = shape_ids(kexp)
        w = np.stack([neg_log2_weights(kexp, sid, owx) for sid in ids])
        t = torch.from_numpy(np.ascontiguousarray(w)).to(device)
        self.cache[key] = (t, ids)
        self.used += t.numel() * 4
        while len(self.cache) > 1 and self.used > self.budget:
            _, old = self.cache.popitem(last=False)
            self.used -= old[0].numel() * 4
        return t, ids


device_weights = DeviceWeights()
