"""Per-point rANS on the CPU -- TEST INFRASTRUCTURE ONLY.

Restates ``latec/rans.py:546-616`` (``rans_encode`` / ``rans_decode`` with one
table row per symbol, picked by the symbol's scale level) on top of the C
coders in ``ans.c``:

* compat: the reference groups the symbols by level and pushes the groups
  last level first, each group with ``encode_reverse``, into one
  constriction ``AnsCoder`` (``latec/rans.py:568-574``); the decoder pops
  level 0 first (``:607-611``). That is one stack coded in reverse over the
  symbols sorted stably by level, which is what ``stack_encode`` does here.
  Byte parity with constriction itself is unpinned (see ``ans.c``).
* native: this project's 32-lane interleaved blob in index order, each lane
  reading its symbol's level row; K symbols per lane from ``lanes_K(n, 4 n)``.
"""

from __future__ import annotations

import numpy as np

from . import ans
from . import rans_model as orm
from .codec import lanes_K


def _wire(kexp, shape, mode):
    cdfs = orm.build_cdfs(kexp, shape)
    return ans.wire_cdfs(cdfs) if mode == "compat" else cdfs


def rans_encode(codes, levels64, radius, kexp=None, shape=0, mode="compat") -> bytes:
    """``latec/rans.py:546-578``."""
    codes = np.asarray(codes, np.uint32).ravel()
    levels = np.asarray(levels64, np.uint8).ravel()
    if codes.shape != levels.shape:
        raise ValueError("codes and levels must have the same flattened length")
    if len(codes) == 0:
        return b""
    if kexp is None:
        kexp = orm.full_kexp(radius)
    syms = orm.narrow(codes, radius, kexp).astype(np.int32)
    cdfs = _wire(kexp, shape, mode)
    if mode == "compat":
        order = np.argsort(levels, kind="stable")
        return ans.stack_encode(syms[order], cdfs, levels[order])
    return ans.lanes_encode(syms, cdfs, lanes_K(len(syms), 4.0 * len(syms)), levels)


def rans_decode(blob: bytes, levels64, radius, kexp=None, shape=0, mode="compat"):
    """``latec/rans.py:581-616``: u32 codes."""
    levels = np.asarray(levels64, np.uint8).ravel()
    n = len(levels)
    if n == 0:
        if blob:
            raise ValueError("non-empty rANS blob for an empty stage")
        return np.empty(0, np.uint32)
    if kexp is None:
        kexp = orm.full_kexp(radius)
    cdfs = _wire(kexp, shape, mode)
    if mode == "compat":
        order = np.argsort(levels, kind="stable")
        syms = np.empty(n, np.int64)
        syms[order] = ans.stack_decode(blob, n, cdfs, levels[order])
    else:
        syms = ans.lanes_decode(blob, n, cdfs, levels).astype(np.int64)
    return orm.widen(syms, radius, kexp).astype(np.uint32)
