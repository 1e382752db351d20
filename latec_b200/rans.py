"""Per-point Laplace-mixture rANS on the device: the learned path's entropy
stage, with the reference's API (``latec/rans.py``).

Every symbol carries its own table row -- the level its predicted Laplacian
scale falls in (``scale_to_level``) -- instead of one level per stage.

* ``mode="compat"`` writes the reference's single-stack byte stream: symbols
  grouped by level (level 0 first, each group in index order) and coded with
  constriction's re-quantised categorical models (``latec/rans.py:546-616``).
  The grouping is a stable counting sort on the device and the coder is the
  device single-stack coder.
* ``mode="native"`` writes this library's interleaved 32-lane blob (the same
  layout as the plain codec's native stages), in index order, each lane
  reading its symbol's level row; it decodes in parallel.

``scale_to_level`` runs on the device by comparing against the 63 float32
level boundaries (found on the host by bisection with the reference formula),
so device and reference levels agree exactly. ``model_bits`` and
``choose_shape`` evaluate the reference's costs on the device in float64.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from functools import lru_cache

import numpy as np

from . import _lib
from . import rans_model as rm
from .rans_model import N_LEVELS, PRECISION, SCALE_HI_MULT, SCALE_LO_DIV, SHAPES

_SELECT_SAMPLE = 0.05   # latec/rans.py: fraction of symbols scored by choose_shape
_SELECT_MIN = 1024      # ... and the least number scored
_PARTIALS = 296         # CTAs of the device cost reductions (2 per SM)


def _torch():
    import torch

    return torch


@dataclass(frozen=True)
class RansTables:
    """``latec/rans.py:17-37``: integer CDFs of the 64-level scale grid of one
    stage eb / radius (the CDFs are eb-invariant), plus the float32 grid."""

    cdfs: np.ndarray
    precision: int
    eb: float
    radius: int
    scale_grid: np.ndarray

    @property
    def total(self) -> int:
        return 1 << self.precision

    @property
    def alphabet(self) -> int:
        return 2 * self.radius

    def cdfs_for(self, kexp: int, shape: int = 0, owx: int = 0) -> np.ndarray:
        return rm.cdfs(int(kexp), int(shape), int(owx), self.cdfs.shape[0], self.precision)


def build_laplace_tables(eb: float, radius: int, *, n_levels: int = N_LEVELS,
                         precision: int = PRECISION) -> RansTables:
    """``latec/rans.py:281-301``."""
    eb, radius = float(eb), int(radius)
    if eb <= 0:
        raise ValueError("eb must be > 0")
    cdfs = rm.cdfs(rm.full_kexp(radius), 0, 0, int(n_levels), int(precision))
    lo, hi = eb / SCALE_LO_DIV, eb * SCALE_HI_MULT
    grid = np.exp(np.linspace(np.log(lo), np.log(hi), int(n_levels))).astype(np.float32)
    return RansTables(cdfs=cdfs, precision=int(precision), eb=eb, radius=radius, scale_grid=grid)


def _scale_to_level_host(scale, eb, n_levels):
    """The reference's float32 formula (``latec/rans.py:270-278``), used only
    to locate the level boundaries."""
    scale = np.asarray(scale, np.float32)
    lo, hi = float(eb) / SCALE_LO_DIV, float(eb) * SCALE_HI_MULT
    t = (np.log(np.clip(scale, lo, hi)) - np.log(lo)) / (np.log(hi) - np.log(lo))
    return np.rint(t * (n_levels - 1)).clip(0, n_levels - 1).astype(np.uint8)


@lru_cache(maxsize=256)
def level_thresholds(eb: float, n_levels: int = N_LEVELS) -> np.ndarray:
    """Float32 boundaries t[k] = the smallest positive float32 whose level is
    k + 1. Positive float32 bit patterns order like the numbers, so a bisection
    over the patterns finds each boundary; a scale's level is then the number
    of boundaries not above it."""
    targets = np.arange(1, n_levels, dtype=np.uint8)
    lo = np.zeros(n_levels - 1, np.uint32)
    hi = np.full(n_levels - 1, np.asarray(np.float32(eb * SCALE_HI_MULT)).view(np.uint32),
                 np.uint32)
    while np.any(lo < hi):
        mid = lo + (hi - lo) // 2
        up = _scale_to_level_host(mid.view(np.float32), eb, n_levels) >= targets
        hi = np.where(up, mid, hi).astype(np.uint32)
        lo = np.where(up, lo, mid + 1).astype(np.uint32)
    return np.ascontiguousarray(lo.view(np.float32))


def _as_device(a, dtype, dev):
    torch = _torch()
    if isinstance(a, torch.Tensor):
        t = a.to(device=dev)
        return t if t.dtype == dtype else t.to(dtype)
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev).to(dtype)


def _device(dev=None):
    torch = _torch()
    return torch.device(dev) if dev is not None else torch.device("cuda",
                                                                 torch.cuda.current_device())


def scale_to_level(scale, eb: float, n_levels: int = N_LEVELS, *, device=None):
    """Quantise Laplacian scales to the shared 64-level log grid on the device
    (``latec/rans.py:270-278``). A CUDA tensor in gives a CUDA uint8 tensor
    out; anything else gives a NumPy uint8 array. NaN scales map to level 0."""
    torch = _torch()
    lib = _lib.load()
    if eb <= 0:
        raise ValueError("eb must be > 0")
    on_dev = isinstance(scale, torch.Tensor) and scale.is_cuda
    dev = scale.device if on_dev else _device(device)
    s = _as_device(scale, torch.float32, dev).contiguous().reshape(-1)
    out = torch.empty(s.numel(), dtype=torch.uint8, device=dev)
    th = level_thresholds(float(eb), int(n_levels))
    arr = (ctypes.c_float * max(len(th), 1))(*th.tolist())
    _lib.check(lib.latec_scale_levels(s.data_ptr(), s.numel(), arr, int(n_levels),
                                      out.data_ptr(), _lib.stream_ptr()), "latec_scale_levels")
    shape = tuple(scale.shape) if hasattr(scale, "shape") else (s.numel(),)
    out = out.reshape(shape)
    return out if on_dev else out.cpu().numpy()


# ------------------------------------------------------------------ internals

def _prep_codes_levels(codes, levels64, tables, dev, kexp=None):
    torch = _torch()
    c = _as_device(codes, torch.int64, dev).reshape(-1)
    lv = _as_device(levels64, torch.int64, dev).reshape(-1)
    if c.shape != lv.shape:
        raise ValueError("codes and levels must have the same flattened length")
    n = c.numel()
    if n:
        if int(c.max()) >= tables.alphabet or int(c.min()) < 0:
            raise ValueError("code exceeds table alphabet")
        if int(lv.max()) >= tables.cdfs.shape[0] or int(lv.min()) < 0:
            raise ValueError("scale level exceeds table count")
        if kexp is not None:  # latec/rans.py:81-88: every bin inside the window
            span = (1 << int(kexp)) - 1
            q = (c - int(tables.radius)).abs()
            if bool(((c != 0) & (q > span)).any()):
                raise ValueError("code outside the narrowed rANS alphabet")
    return c.to(torch.int16), lv.to(torch.uint8), n


def _level_order(lv, n, dev):
    torch = _torch()
    lib = _lib.load()
    order = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    ws = torch.empty(int(lib.latec_level_order_workspace_bytes(n)), dtype=torch.uint8, device=dev)
    _lib.check(lib.latec_level_order(lv.data_ptr(), n, order.data_ptr(), ws.data_ptr(), ws.numel(),
                                     _lib.stream_ptr()), "latec_level_order")
    return order


def _permute(src, order, n, inverse=False):
    torch = _torch()
    lib = _lib.load()
    dst = torch.empty_like(src)
    _lib.check(lib.latec_permute(src.data_ptr(), src.element_size(), order.data_ptr(), n,
                                 dst.data_ptr(), int(inverse), _lib.stream_ptr()), "latec_permute")
    return dst


def _mode_id(mode):
    if mode == "compat":
        return _lib.RANS_COMPAT
    if mode == "native":
        return _lib.RANS_LANES
    raise ValueError("mode must be 'compat' or 'native'")


def rans_encode(codes, levels64, tables: RansTables, *, kexp: int | None = None, shape: int = 0,
                mode: str = "compat", device=None) -> bytes:
    """Entropy-code ``codes`` (u32 bins, 0 = outlier) with per-point table rows
    ``levels64`` (``latec/rans.py:546-578``). Returns the blob bytes."""
    torch = _torch()
    lib = _lib.load()
    mid = _mode_id(mode)
    dev = _device(device)
    if kexp is None:
        kexp = rm.full_kexp(tables.radius)
    kexp, shape = int(kexp), int(shape)
    c, lv, n = _prep_codes_levels(codes, levels64, tables, dev, kexp)
    if n == 0:
        return b""
    if mid == _lib.RANS_COMPAT:
        order = _level_order(lv, n, dev)
        c, lv = _permute(c, order, n), _permute(lv, order, n)
    cdf, enc, bucket, alphabet = rm.device_tables.get(mid, kexp, shape, 0, None, dev)
    stages = (_lib.RansStage * 1)()
    d = stages[0]
    d.codes_off = d.out_off = 0
    d.n = n
    d.kexp, d.radius, d.mode, d.per_point = kexp, int(tables.radius), mid, 1
    d.alphabet = alphabet
    d.framed_hi = 0
    d.cdf, d.enc, d.bucket = cdf.data_ptr(), enc.data_ptr(), bucket.data_ptr()
    d.K = rm.lanes_K(n, 4.0 * n) if mid == _lib.RANS_LANES else 0
    wsb = lib.latec_rans_encode_workspace_bytes(stages, 1)
    ws = torch.empty(max(int(wsb), 1), dtype=torch.uint8, device=dev)
    cap = (16 + 4 * (1 + 65 * d.n_chunks + n + 2) + 15) // 16 * 16
    payload = torch.empty(cap, dtype=torch.uint8, device=dev)
    plen = torch.zeros(1, dtype=torch.int64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    stats = torch.zeros(ctypes.sizeof(_lib.StageStats), dtype=torch.uint8, device=dev)
    _lib.check(lib.latec_rans_encode(stages, 1, c.data_ptr(), lv.data_ptr(), stats.data_ptr(),
                                     None, 4, payload.data_ptr(), cap, plen.data_ptr(),
                                     err.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream_ptr()),
               "latec_rans_encode")
    if int(err.item()):
        raise RuntimeError(f"entropy coder reported error bits {int(err.item()):#x}")
    rec = payload[:int(plen.item())].cpu().numpy().tobytes()
    # stage record: u32 n | u64 frame | blob | u32 n_out
    hlen = int.from_bytes(rec[4:12], "little") & ((1 << 45) - 1)
    return rec[12:12 + hlen]


def rans_decode(blob: bytes, levels64, tables: RansTables, *, kexp: int | None = None,
                shape: int = 0, mode: str = "compat", device=None) -> np.ndarray:
    """Inverse of ``rans_encode`` (``latec/rans.py:581-616``): u32 codes."""
    torch = _torch()
    lib = _lib.load()
    mid = _mode_id(mode)
    dev = _device(device)
    lv = _as_device(levels64, torch.int64, dev).reshape(-1)
    n = lv.numel()
    if n == 0:
        if blob:
            raise ValueError("non-empty rANS blob for an empty stage")
        return np.empty(0, np.uint32)
    if len(blob) % 4:
        raise ValueError("rANS payload is not aligned to 32-bit words")
    if int(lv.max()) >= tables.cdfs.shape[0] or int(lv.min()) < 0:
        raise ValueError("scale level exceeds table count")
    lv = lv.to(torch.uint8)
    if kexp is None:
        kexp = rm.full_kexp(tables.radius)
    kexp, shape = int(kexp), int(shape)
    words_np = np.frombuffer(bytes(blob), "<u4")
    order = None
    if mid == _lib.RANS_COMPAT:
        order = _level_order(lv, n, dev)
        lv = _permute(lv, order, n)
    cdf, enc, bucket, alphabet = rm.device_tables.get(mid, kexp, shape, 0, None, dev)
    stages = (_lib.RansStage * 1)()
    d = stages[0]
    d.codes_off, d.n = 0, n
    d.kexp, d.radius, d.mode, d.per_point = kexp, int(tables.radius), mid, 1
    d.alphabet = alphabet
    d.cdf, d.enc, d.bucket = cdf.data_ptr(), enc.data_ptr(), bucket.data_ptr()
    d.blob_off, d.blob_words = 0, len(words_np)
    ranges = None
    total_chunks = 0
    if mid == _lib.RANS_LANES:
        if len(words_np) < 1 or int(words_np[0]) < 1:
            raise ValueError("malformed rANS payload")
        K = int(words_np[0])
        nc = -(-n // (32 * K))
        if len(words_np) < 1 + nc:
            raise ValueError("malformed rANS payload")
        sizes = words_np[1:1 + nc].astype(np.int64)
        ends = 1 + nc + np.cumsum(sizes)
        if int(ends[-1]) != len(words_np):
            raise ValueError("trailing data in rANS payload")
        starts = ends - sizes
        ranges = _as_device(np.stack([starts, ends], 1).reshape(-1), torch.int64, dev)
        d.K, d.n_chunks, d.chunk0 = K, nc, 0
        total_chunks = nc
    words = torch.from_numpy(np.concatenate([words_np, np.zeros(2, np.uint32)]).view(np.int32))
    words = words.to(dev)
    codes = torch.empty(n, dtype=torch.int16, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    ws = torch.empty(int(lib.latec_rans_decode_workspace_bytes(1)), dtype=torch.uint8, device=dev)
    _lib.check(lib.latec_rans_decode(stages, 1, total_chunks, words.data_ptr(),
                                     ranges.data_ptr() if ranges is not None else None,
                                     lv.data_ptr(), codes.data_ptr(), err.data_ptr(), ws.data_ptr(),
                                     ws.numel(), _lib.stream_ptr()), "latec_rans_decode")
    e = int(err.item())
    if e & (4 | 8):
        raise ValueError("trailing data in rANS payload")
    if e:
        raise ValueError(f"malformed rANS payload (error bits {e:#x})")
    if order is not None:
        codes = _permute(codes, order, n, inverse=True)
    return codes.cpu().numpy().view(np.uint16).astype(np.uint32)


def model_bits(codes, levels64, tables: RansTables, *, kexp: int | None = None,
               shape: int = 0, device=None) -> float:
    """Ideal coded length in bits under the per-point tables
    (``latec/rans.py:332-357``), summed in float64 on the device."""
    torch = _torch()
    lib = _lib.load()
    dev = _device(device)
    if kexp is None:
        kexp = rm.full_kexp(tables.radius)
    c, lv, n = _prep_codes_levels(codes, levels64, tables, dev, kexp)
    if n == 0:
        return 0.0
    cdf, _enc, _bucket, alphabet = rm.device_tables.get(_lib.RANS_LANES, int(kexp), int(shape), 0,
                                                        None, dev)
    part = torch.zeros(_PARTIALS, dtype=torch.float64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.latec_point_bits(c.data_ptr(), lv.data_ptr(), n, cdf.data_ptr(), alphabet,
                                    int(tables.radius), int(kexp), part.data_ptr(), _PARTIALS,
                                    err.data_ptr(), _lib.stream_ptr()), "latec_point_bits")
    if int(err.item()):
        raise ValueError("code outside the stage window")
    return float(math.fsum(part.cpu().numpy().tolist()))


def choose_shape(codes, levels64, tables: RansTables, kexp: int, *,
                 sample: float = _SELECT_SAMPLE, device=None) -> int:
    """Dictionary entry minimising the stage's coded length, scored on a
    strided sample against the continuous per-level weights
    (``latec/rans.py:204-243``); costs are float64 sums on the device."""
    dev = _device(device)
    c, lv, n = _prep_codes_levels(codes, levels64, tables, dev, kexp)
    if n == 0:
        return 0
    ids, part = shape_costs(c.data_ptr(), lv.data_ptr(), n, tables, kexp, dev, sample)
    return pick_shape(ids, part.cpu().numpy())


def shape_costs(codes_ptr, levels_ptr, n, tables: RansTables, kexp: int, dev,
                sample: float = _SELECT_SAMPLE):
    """Launch ``choose_shape``'s cost sums for n int16 codes and uint8 level
    rows at the given device addresses (n > 0); returns the candidate ids
    and the device partial sums for ``pick_shape``."""
    torch = _torch()
    lib = _lib.load()
    n_levels = tables.cdfs.shape[0]
    step = 1
    if sample < 1.0:
        step = max(1, n // max(_SELECT_MIN, int(n * sample)))
    w = rm.level_weights(int(kexp), n_levels)
    wt = _as_device(w, torch.float64, dev).contiguous()
    ids = rm.shape_ids(int(kexp))
    ds = (ctypes.c_int32 * len(ids))(*[SHAPES[i][0] for i in ids])
    ws = (ctypes.c_double * len(ids))(*[SHAPES[i][1] for i in ids])
    part = torch.zeros(len(ids) * _PARTIALS, dtype=torch.float64, device=dev)
    _lib.check(lib.latec_shape_costs(codes_ptr, levels_ptr, n, step, wt.data_ptr(),
                                     w.shape[1], n_levels, int(tables.radius), int(kexp),
                                     1.0 / tables.total, ds, ws, len(ids), part.data_ptr(),
                                     _PARTIALS, _lib.stream_ptr()), "latec_shape_costs")
    return ids, part


def pick_shape(ids, partials) -> int:
    """The candidate with the least cost (fsum of its partial sums; the first
    one on ties)."""
    costs = np.asarray(partials).reshape(len(ids), _PARTIALS)
    best_id, best = 0, math.inf
    for k, sid in enumerate(ids):
        cost = math.fsum(costs[k].tolist())
        if cost < best:
            best_id, best = sid, cost
    return best_id
