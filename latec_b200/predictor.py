"""``InterpPredictor``: the SZ3-style interpolation plugin, evaluated on the GPU.

Same constructor, attributes and ``predict(recon, known, pos)`` contract as the
reference (``latec/predictor.py:159-317``); the codec recognises it and runs
its stages through the fused CUDA kernels, and a direct ``predict`` call runs
the prediction-only kernel for the stage that ``known`` identifies.
"""

from __future__ import annotations

import ctypes
import itertools

import numpy as np

from . import _lib
from .bitstream import FLAG_CUBIC, FLAG_INTERP

END_QUAD = 1 << 0
END_EXTRAP = 1 << 1
END_MODE_MAX = END_QUAD | END_EXTRAP


def default_interp_center(ndim: int) -> int:
    """``latec/predictor.py:21-27``: average the odd axes up to 3-D, first axis from 4-D."""
    return 1 if ndim >= 4 else 0


def default_interp_end_mode(ndim: int) -> int:
    """``latec/predictor.py:51-66``: quadratic line ends."""
    return END_QUAD


class LazyStageMasks:
    """The schedule's boolean stage masks, built one at a time on the host
    (``latec/levels.py:150-177``); the CUDA codec never needs them."""

    def __init__(self, shape, levels, anchor_stride, anchor_block=1):
        from .levels import check_plan

        self.shape = check_plan(shape, levels, anchor_stride, anchor_block)
        self.levels, self.anchor_stride, self.anchor_block = levels, anchor_stride, anchor_block

    def __len__(self):
        return 1 + self.levels * (2 * len(self.shape) - 1)

    def __iter__(self):
        shape, nd = self.shape, len(self.shape)
        covered = np.zeros(shape, bool)
        m = np.zeros(shape, bool)
        for offs in itertools.product(range(self.anchor_block), repeat=nd):
            m[tuple(slice(o, None, self.anchor_stride) for o in offs)] = True
        covered |= m
        yield m
        for k in range(1, self.levels + 1):
            s = max(self.anchor_stride >> k, 1)

            def sl(odd):
                return tuple(slice(s, None, 2 * s) if j in odd else slice(0, None, 2 * s)
                             for j in range(nd))

            for axis in range(nd):
                m = np.zeros(shape, bool)
                m[sl((axis,))] = True
                m &= ~covered
                if k == self.levels and nd == 1:
                    m |= ~covered
                covered |= m
                yield m
            for w in range(2, nd + 1):
                m = np.zeros(shape, bool)
                for axes in itertools.combinations(range(nd), w):
                    m[sl(axes)] = True
                m &= ~covered
                if k == self.levels and w == nd:
                    m |= ~covered
                covered |= m
                yield m


class InterpPredictor:
    """SZ3-style cubic/linear interpolation over the dyadic schedule."""

    _latec_gpu_interp = True  # the codec runs this predictor's stages in CUDA
    tunable = True
    fast_eb_ratio = 0.9

    def __init__(self, order: str = "cubic", levels: int = 4, anchor_stride: int = 16,
                 anchor_block: int = 4, center: int | None = None, end_mode: int | None = None):
        if order not in ("linear", "cubic"):
            raise ValueError("order must be 'linear' or 'cubic'")
        if end_mode is not None and not 0 <= end_mode <= END_MODE_MAX:
            raise ValueError(f"end_mode must be in [0, {END_MODE_MAX}]")
        self.order = order
        self.levels = levels
        self.anchor_stride = anchor_stride
        self.anchor_block = anchor_block
        self.center = center
        self.end_mode = end_mode
        self.stream_flag = FLAG_INTERP | (FLAG_CUBIC if order == "cubic" else 0)
        self.checkpoint_hash = b"\0" * 16

    def stage_masks(self, shape, levels, anchor_stride, anchor_block):
        return LazyStageMasks(shape, levels, anchor_stride, anchor_block)

    def predict(self, recon, known, pos=None):
        """Prediction at the stage ``pos`` that follows the points in ``known``.

        ``recon`` is ``(C, *S)`` (NumPy or torch, host or CUDA); returns the
        compact ``(C, pos.sum())`` prediction (float32, float64 for a float64
        reconstruction) in the same kind as ``recon``."""
        import torch

        from .levels import plan_for

        if pos is None:
            raise NotImplementedError("predict needs the stage mask `pos`")
        is_t = isinstance(recon, torch.Tensor)
        shape = tuple(recon.shape[1:])
        plan = plan_for(shape, self.levels, self.anchor_stride, self.anchor_block)
        nk = int(known.sum()) if not isinstance(known, torch.Tensor) else int(known.sum().item())
        covered, stage = 0, None
        for t, n in enumerate(plan.counts):
            if t > 0 and n and covered == nk:
                stage = t
                break
            covered += n
        if stage is None:
            raise ValueError("known mask does not match the interp schedule")
        npos = int(pos.sum()) if not isinstance(pos, torch.Tensor) else int(pos.sum().item())
        if npos != plan.counts[stage]:
            raise ValueError("pos does not match the interp schedule")
        center = self.center if self.center is not None else default_interp_center(len(shape))
        end_mode = self.end_mode if self.end_mode is not None else default_interp_end_mode(len(shape))
        dev = recon.device if (is_t and recon.is_cuda) else torch.device("cuda")
        r = recon if is_t else torch.from_numpy(np.ascontiguousarray(recon))
        f64 = r.dtype == torch.float64
        r = r.to(dev, torch.float64 if f64 else torch.float32).contiguous()
        c = int(r.shape[0])
        out = torch.empty((c, npos), dtype=r.dtype, device=dev)
        prm = _lib.QuantParams(dtype=_lib.F64 if f64 else _lib.F32, channels=c, radius=1,
                               order=1 if self.order == "cubic" else 0, center=int(center),
                               end_mode=int(end_mode), round_output=0, reserved=0)
        lib = _lib.load()
        _lib.check(lib.latec_interp_predict_stage(plan.handle, stage, ctypes.byref(prm),
                                                  r.data_ptr(), out.data_ptr(), _lib.stream_ptr()),
                   "latec_interp_predict_stage")
        if is_t and recon.is_cuda:
            return out
        return out.cpu().numpy()
