"""Dyadic stage schedule on the host: the plan handle of the CUDA library plus
the closed-form helpers the codec needs (reference ``latec/levels.py``).

The plan is built in C++ (``latec_plan_create``) from the header parameters
alone -- no stage mask is ever materialised; the kernels decode each stage's
points from its rank.
"""

from __future__ import annotations

import ctypes
import threading
from collections import OrderedDict

import numpy as np

from . import _lib


def check_plan(shape, levels, anchor_stride, anchor_block):
    """Parameter validation with the reference's messages (``latec/levels.py:54-76``)."""
    shape = tuple(int(n) for n in shape)
    if len(shape) < 1:
        raise ValueError("shape must have at least one axis")
    if levels < 1:
        raise ValueError("levels must be >= 1")
    if anchor_stride < 2 or anchor_stride & (anchor_stride - 1):
        raise ValueError("anchor_stride must be a power of two >= 2")
    if not 1 <= anchor_block <= anchor_stride:
        raise ValueError("anchor_block must be in [1, anchor_stride]")
    if (1 << levels) < anchor_stride:
        raise ValueError(
            f"levels={levels} too small for anchor_stride={anchor_stride}: need levels >= "
            f"log2(anchor_stride) = {anchor_stride.bit_length() - 1} to densify to stride 1")
    return shape


def n_stages(ndim, levels):
    return 1 + levels * (2 * ndim - 1)


def stage_strides(ndim, levels, anchor_stride):
    out = [anchor_stride]
    for k in range(1, levels + 1):
        out += [max(anchor_stride >> k, 1)] * (2 * ndim - 1)
    return out


def stage_ebs(shape, levels, anchor_stride, anchor_block, eb, eb_ratio):
    """``eb * eb_ratio ** log2(stride / finest)`` per stage, evaluated with the
    same NumPy float64 expression as ``latec/levels.py:382-386``."""
    strides = stage_strides(len(shape), levels, anchor_stride)
    if not 1 <= anchor_block <= anchor_stride:
        raise ValueError("anchor_block must be in [1, anchor_stride]")
    finest = min(strides)
    return [eb * eb_ratio ** np.log2(s / finest) for s in strides]


class Plan:
    """Owner of a ``latec_plan`` handle for one (shape, levels, stride) schedule."""

    def __init__(self, shape, levels, anchor_stride, anchor_block=1):
        self.shape = check_plan(shape, levels, anchor_stride, anchor_block)
        if len(self.shape) > 6:
            raise NotImplementedError("the CUDA schedule supports up to 6 spatial axes")
        self.levels, self.anchor_stride, self.anchor_block = levels, anchor_stride, anchor_block
        lib = _lib.load(require_gpu=False)
        arr = (ctypes.c_uint32 * len(self.shape))(*self.shape)
        h = ctypes.c_void_p()
        _lib.check(lib.latec_plan_create(arr, len(self.shape), levels, anchor_stride, anchor_block,
                                         ctypes.byref(h)), "latec_plan_create")
        self._h = h
        self._lib = lib
        ns = lib.latec_plan_num_stages(h)
        self.counts, self.strides, self.weights, self.axes = [], [], [], []
        for t in range(ns):
            n, s, w, a = ctypes.c_uint64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
            _lib.check(lib.latec_plan_stage_info(h, t, ctypes.byref(n), ctypes.byref(s),
                                                 ctypes.byref(w), ctypes.byref(a)))
            self.counts.append(int(n.value))
            self.strides.append(int(s.value))
            self.weights.append(int(w.value))
            self.axes.append(int(a.value))

    @property
    def handle(self):
        return self._h

    def __len__(self):
        return len(self.counts)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.latec_plan_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._h = None


_plans: "OrderedDict" = OrderedDict()
_plans_lock = threading.Lock()
_PLAN_CACHE = 1024  # schedules kept (host memory only, a few KB each)


def plan_for(shape, levels, anchor_stride, anchor_block=1) -> Plan:
    """The schedule of a shape, from a least-recently-used cache: a batch of
    many tensors of different shapes reuses its plans from call to call.
    Safe to call from several host threads: the cache is updated under a
    lock, and a plan built concurrently by two threads is kept once."""
    key = (tuple(int(n) for n in shape), int(levels), int(anchor_stride), int(anchor_block))
    with _plans_lock:
        p = _plans.get(key)
        if p is not None:
            _plans.move_to_end(key)
            return p
    built = Plan(*key)  # outside the lock: the C++ plan build may take a while
    with _plans_lock:
        p = _plans.setdefault(key, built)
        _plans.move_to_end(key)
        while len(_plans) > _PLAN_CACHE:
            _plans.popitem(last=False)
    return p


def stage_counts(shape, levels, anchor_stride, anchor_block=1):
    """Closed-form stage sizes (``latec/levels.py:221-282``) from the C++ plan."""
    return list(plan_for(shape, levels, anchor_stride, anchor_block).counts)
