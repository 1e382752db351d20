"""ctypes binding of the C oracle coder (``oracle/ans.c``) -- test infrastructure only."""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liblatec_oracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "ans.c")
        if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", _HERE])
        L = ctypes.CDLL(_SO)
        P = ctypes.c_void_p
        L.oracle_fast_quantize.argtypes = [P, ctypes.c_int, P]
        L.oracle_fast_quantize.restype = ctypes.c_int
        for name in ("oracle_stack_encode",):
            f = getattr(L, name)
            f.argtypes = [P, P, ctypes.c_long, P, ctypes.c_int, P, ctypes.c_long]
            f.restype = ctypes.c_long
        L.oracle_lanes_encode.argtypes = [P, P, ctypes.c_long, ctypes.c_int, P, ctypes.c_int, P,
                                          ctypes.c_long]
        L.oracle_lanes_encode.restype = ctypes.c_long
        for name in ("oracle_stack_decode", "oracle_lanes_decode"):
            f = getattr(L, name)
            f.argtypes = [P, ctypes.c_long, P, ctypes.c_long, P, ctypes.c_int, P]
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def fast_quantize(probs):
    """constriction's float32 fast quantisation -> wire CDF (n + 1,) uint32."""
    probs = np.ascontiguousarray(probs, np.float32)
    out = np.empty(len(probs) + 1, np.uint32)
    rc = lib().oracle_fast_quantize(_p(probs), len(probs), _p(out))
    if rc:
        raise ValueError(f"fast quantisation failed ({rc})")
    return out


def wire_cdfs(cdfs):
    """Per-row fast re-quantisation of integer CDF rows (compat model)."""
    cdfs = np.asarray(cdfs)
    out = np.empty(cdfs.shape, np.uint32)
    for r in range(cdfs.shape[0]):
        out[r] = fast_quantize(np.diff(cdfs[r].astype(np.int64)).astype(np.float32))
    return out


def _prep(syms, levels, cdfs):
    syms = np.ascontiguousarray(syms, np.int32)
    lv = None if levels is None else np.ascontiguousarray(levels, np.uint8)
    cdfs = np.ascontiguousarray(cdfs, np.uint32)
    if cdfs.ndim == 1:
        cdfs = cdfs[None]
    return syms, lv, cdfs, cdfs.shape[1] - 1


def stack_encode(syms, cdfs, levels=None) -> bytes:
    syms, lv, cdfs, alphabet = _prep(syms, levels, cdfs)
    cap = len(syms) + 4
    out = np.empty(cap, np.uint32)
    n = lib().oracle_stack_encode(_p(syms), _p(lv), len(syms), _p(cdfs), alphabet, _p(out), cap)
    if n < 0:
        raise ValueError(f"stack encode failed ({n})")
    return out[:n].astype("<u4").tobytes()


def stack_decode(blob: bytes, n, cdfs, levels=None):
    words = np.frombuffer(blob, "<u4").astype(np.uint32)
    _, lv, cdfs, alphabet = _prep(np.zeros(0), levels, cdfs)
    out = np.empty(n, np.int32)
    rc = lib().oracle_stack_decode(_p(words), len(words), _p(lv), n, _p(cdfs), alphabet, _p(out))
    if rc:
        raise ValueError(f"stack decode failed ({rc})")
    return out


def lanes_encode(syms, cdfs, K, levels=None) -> bytes:
    syms, lv, cdfs, alphabet = _prep(syms, levels, cdfs)
    per = 32 * K
    n_chunks = (len(syms) + per - 1) // per
    cap = 1 + n_chunks + len(syms) + 64 * n_chunks + 4
    out = np.empty(cap, np.uint32)
    n = lib().oracle_lanes_encode(_p(syms), _p(lv), len(syms), int(K), _p(cdfs), alphabet,
                                  _p(out), cap)
    if n < 0:
        raise ValueError(f"lanes encode failed ({n})")
    return out[:n].astype("<u4").tobytes()


def lanes_decode(blob: bytes, n, cdfs, levels=None):
    words = np.frombuffer(blob, "<u4").astype(np.uint32)
    _, lv, cdfs, alphabet = _prep(np.zeros(0), levels, cdfs)
    out = np.empty(n, np.int32)
    rc = lib().oracle_lanes_decode(_p(words), len(words), _p(lv), n, _p(cdfs), alphabet, _p(out))
    if rc:
        raise ValueError(f"lanes decode failed ({rc})")
    return out
