"""Oracle restatement of the Laplace-mixture rANS model (reference ``latec/rans.py``).

Test infrastructure only (see ``oracle/__init__.py``). Everything here is
deterministic NumPy: the per-level continuous weights, the 21-entry mixture
dictionary, the outlier-marker weights, the 24-bit integer PMF quantisation,
the stage-constant level fit and the per-point shape pick.
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np

SCALE_LO_DIV = 16.0
SCALE_HI_MULT = 4096.0
N_LEVELS = 64
PRECISION = 24
# latec/rans.py:119-127
SHAPES = ((0, 0.0),) + tuple((d, w) for d in (4, 8, 16, 24) for w in (0.02, 0.05, 0.12, 0.25, 0.45))
# latec/rans.py:148-157
OUTLIER_WEIGHTS = (0.0, 2.0**-13, 2.0**-10, 2.0**-8, 2.0**-6, 2.0**-4, 2.0**-2, 0.5)
_WIDE_KEXP = 13
_CONST_TILE = 1 << 22


def full_kexp(radius):
    """``latec/rans.py:65-67``."""
    return max(1, int(int(radius) - 1).bit_length())


def choose_kexp(codes, radius):
    """``latec/rans.py:70-80``."""
    codes = np.asarray(codes, np.uint32).ravel()
    inr = codes[codes != 0]
    if len(inr) == 0:
        return 1
    return max(1, int(np.abs(inr.astype(np.int64) - int(radius)).max()).bit_length())


def narrow(codes, radius, kexp):
    """``latec/rans.py:83-90``."""
    span = (1 << int(kexp)) - 1
    q = np.asarray(codes).astype(np.int64) - int(radius)
    syms = np.where(np.asarray(codes) == 0, 0, q + span + 1)
    if len(syms) and (int(syms.min()) < 0 or int(syms.max()) > 2 * span + 1):
        raise ValueError("code outside the narrowed rANS alphabet")
    return syms


def widen(syms, radius, kexp):
    """``latec/rans.py:93-97``."""
    span = (1 << int(kexp)) - 1
    codes = np.asarray(syms).astype(np.int64) - span - 1 + int(radius)
    return np.where(np.asarray(syms) == 0, 0, codes).astype(np.uint32)


def shape_ids(kexp):
    """``latec/rans.py:194-201``."""
    if kexp < _WIDE_KEXP:
        return tuple(range(len(SHAPES)))
    return (0,) + tuple(i for i, (_d, w) in enumerate(SHAPES) if w == 0.02)


def _laplace_cdf(x, b):
    """``latec/rans.py:667-669``."""
    z = np.clip(x / b, -700.0, 700.0)
    return np.where(x < 0, 0.5 * np.exp(z), 1.0 - 0.5 * np.exp(-z))


@lru_cache(maxsize=32)
def level_weights(kexp, n_levels=N_LEVELS):
    """``latec/rans.py:246-267``."""
    span = (1 << kexp) - 1
    alphabet = 2 * span + 2
    eb = 1.0
    lo, hi = eb / SCALE_LO_DIV, eb * SCALE_HI_MULT
    grid = np.exp(np.linspace(np.log(lo), np.log(hi), n_levels)).astype(np.float64)
    q = np.arange(-span, span + 1, dtype=np.float64)
    left = q * (2.0 * eb) - eb
    right = q * (2.0 * eb) + eb
    w = np.empty((n_levels, alphabet), np.float64)
    for i, b in enumerate(grid):
        w[i, 1:] = _laplace_cdf(right, b) - _laplace_cdf(left, b)
        w[i, 0] = w[i, 1:].max() * 1e-9
    w /= w.sum(1, keepdims=True)
    return w


@lru_cache(maxsize=256)
def shaped_weights(kexp, shape, n_levels=N_LEVELS):
    """``latec/rans.py:376-384``."""
    weights = level_weights(kexp, n_levels)
    d, w = SHAPES[shape]
    if not w:
        return weights
    broad = weights[np.minimum(np.arange(n_levels) + d, n_levels - 1)]
    return (1.0 - w) * weights + w * broad


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
    """Largest-remainder quantisation to counts summing to ``total``, every
    count >= 1; ``latec/rans.py:676-722``."""
    w = np.asarray(weights, np.float64)
    n_rows, alphabet = w.shape
    scaled = w / w.sum(1, keepdims=True) * total
    floor = np.floor(scaled)
    pmf = np.maximum(floor.astype(np.int64), 1)
    frac = scaled - floor
    diff = total - pmf.sum(1)
    up = np.flatnonzero(diff > 0)
    if len(up):
        d = diff[up]
        bulk, rem = np.divmod(d, alphabet)
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
def build_cdfs(kexp, shape=0, n_levels=N_LEVELS, precision=PRECISION, owx=0):
    """``(n_levels, alphabet + 1)`` uint32 CDFs; ``latec/rans.py:304-329``."""
    span = (1 << kexp) - 1
    alphabet = 2 * span + 2
    total = 1 << precision
    weights = with_outlier_weight(shaped_weights(kexp, shape, n_levels), owx)
    cdfs = np.empty((n_levels, alphabet + 1), np.uint32)
    cdfs[:, 0] = 0
    cdfs[:, 1:] = np.cumsum(quantize_pmf_rows(weights, total), axis=1, dtype=np.uint64)
    return cdfs


@lru_cache(maxsize=256)
def neg_log2_weights(kexp, shape, n_levels=N_LEVELS, precision=PRECISION, owx=0):
    """``latec/rans.py:387-392``."""
    weights = with_outlier_weight(shaped_weights(kexp, shape, n_levels), owx)
    floor = 1.0 / (1 << precision)
    return -np.log2(np.maximum(weights, floor)).astype(np.float32)


def choose_outlier_weight(n_outliers, n_codes):
    """``latec/rans.py:162-169``."""
    if n_codes <= 0 or n_outliers <= 0:
        return 0
    rate = n_outliers / n_codes
    return int(np.argmin([abs(np.log(max(w, 1e-12)) - np.log(rate)) for w in OUTLIER_WEIGHTS]))


def const_hist(codes, radius, kexp):
    """float32 symbol histogram accumulated per 2^22-code tile, exactly as
    ``latec/rans.py:414-420`` does (float32 += int64 bincount)."""
    codes = np.asarray(codes, np.uint32).ravel()
    alphabet = 2 * ((1 << int(kexp)) - 1) + 2
    hist = np.zeros(alphabet, np.float32)
    for a in range(0, len(codes), _CONST_TILE):
        hist += np.bincount(narrow(codes[a:a + _CONST_TILE], radius, kexp), minlength=alphabet)
    return hist


def choose_const_level_from_hist(hist, n_codes, kexp, n_levels=N_LEVELS, precision=PRECISION):
    """Level/shape/outlier-weight argmin over the f32 histogram;
    ``latec/rans.py:421-430``."""
    owx = choose_outlier_weight(int(hist[0]), n_codes)
    best = (np.inf, 0, 0)
    for sid in shape_ids(int(kexp)):
        cost = neg_log2_weights(int(kexp), int(sid), n_levels, precision, owx) @ hist
        level = int(cost.argmin())
        if cost[level] < best[0]:
            best = (float(cost[level]), level, int(sid))
    return best[1], best[2], owx, best[0]


def choose_const_level(codes, radius, kexp):
    """``latec/rans.py:395-430``."""
    codes = np.asarray(codes, np.uint32).ravel()
    if len(codes) == 0:
        return 0, 0, 0, 0.0
    return choose_const_level_from_hist(const_hist(codes, radius, kexp), len(codes), kexp)


def scale_grid(eb, n_levels=N_LEVELS):
    """``latec/rans.py:296-298``."""
    lo, hi = eb / SCALE_LO_DIV, eb * SCALE_HI_MULT
    return np.exp(np.linspace(np.log(lo), np.log(hi), n_levels)).astype(np.float32)


def scale_to_level(scale, eb, n_levels=N_LEVELS):
    """``latec/rans.py:270-278``."""
    scale = np.asarray(scale, np.float32)
    lo, hi = float(eb) / SCALE_LO_DIV, float(eb) * SCALE_HI_MULT
    t = (np.log(np.clip(scale, lo, hi)) - np.log(lo)) / (np.log(hi) - np.log(lo))
    return np.rint(t * (n_levels - 1)).clip(0, n_levels - 1).astype(np.uint8)


def choose_shape(codes, levels64, radius, kexp, sample=0.05, n_levels=N_LEVELS,
                 precision=PRECISION):
    """``latec/rans.py:204-243``."""
    codes = np.asarray(codes, np.uint32).ravel()
    if len(codes) == 0:
        return 0
    syms = narrow(codes, radius, kexp)
    levels = np.asarray(levels64, np.uint8).ravel().astype(np.int64)
    if sample < 1.0:
        step = max(1, len(syms) // max(1024, int(len(syms) * sample)))
        if step > 1:
            syms, levels = syms[::step], levels[::step]
    weights = level_weights(int(kexp), n_levels)
    floor = 1.0 / (1 << precision)
    idx = np.arange(n_levels)
    best_id, best_cost = 0, np.inf
    for sid in shape_ids(int(kexp)):
        d, w = SHAPES[sid]
        p = weights[levels, syms]
        if w:
            broad = weights[np.minimum(idx + d, n_levels - 1)[levels], syms]
            p = (1.0 - w) * p + w * broad
        cost = -np.log2(np.maximum(p, floor)).sum()
        if cost < best_cost:
            best_id, best_cost = sid, float(cost)
    return best_id


def model_bits(codes, levels64, radius, kexp, shape=0):
    """``latec/rans.py:332-357``."""
    codes = np.asarray(codes, np.uint32).ravel()
    levels = np.asarray(levels64, np.uint8).ravel()
    if len(codes) == 0:
        return 0.0
    cdfs = build_cdfs(kexp, shape)
    syms = narrow(codes, radius, kexp)
    probs = np.empty(len(codes), np.float64)
    for level in range(cdfs.shape[0]):
        idx = np.flatnonzero(levels == level)
        if len(idx):
            s = syms[idx]
            cdf = cdfs[level]
            probs[idx] = cdf[s + 1].astype(np.int64) - cdf[s].astype(np.int64)
    return float((-np.log2(probs / (1 << PRECISION))).sum())


FIT_FRAC_BITS = 20  # fixed-point fraction bits of the native fit's weights


def fit_const_native(counts, n_codes, kexp, n_levels=N_LEVELS, precision=PRECISION):
    """Stage-constant fit of the native entropy mode: the reference's model
    space and selection rule (``latec/rans.py:421-430``: first minimum over
    levels, then the first strictly smaller cost over shapes) with every cost
    an exact integer, sum over the alphabet of ``Wq[level, sym] * count[sym]``
    where ``Wq = rint(W * 2^20)`` of the float32 weights ``W`` (-log2 p); the
    returned cost in bits is ``float(sum) * 2^-20``."""
    counts = np.asarray(counts, np.int64)
    owx = choose_outlier_weight(int(counts[0]), n_codes)
    best = (None, 0, 0)
    for sid in shape_ids(int(kexp)):
        w = neg_log2_weights(int(kexp), int(sid), n_levels, precision, owx)
        wq = np.rint(w.astype(np.float64) * float(1 << FIT_FRAC_BITS)).astype(np.int64)
        cost = wq @ counts  # exact: every partial sum stays below 2^56
        level = int(np.argmin(cost))  # the first minimum
        if best[0] is None or int(cost[level]) < best[0]:
            best = (int(cost[level]), level, int(sid))
    return best[1], best[2], owx, float(best[0]) * 2.0 ** -FIT_FRAC_BITS
