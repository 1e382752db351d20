"""``GNNCodec``: the learned LATEC codec on the device (``latec/gnn_codec.py``).

Same API as the reference codec: ``GNNCodec(checkpoint_path, device=None, *,
strict_checkpoint=True)``, ``compress(x, error_bound, ...) -> bytes`` and
``uncompress(stream) -> torch.Tensor`` (alias ``decompress``), and the same
stream container: ``<8sII`` prefix (magic ``LATECGNN``, version, header
length), a JSON metadata header, then a zstd frame of the stage payload
(``latec/gnn_codec.py:229-246``).

The tensor is min-max normalised to [0, 1] in float32 and ``error_bound`` is
applied to the normalised values, so it is relative to the data range, as in
the reference (``:1509-1522``). Each stage of the dyadic schedule is coded as
follows.

1. The GNN predicts (mu, log2 b) at the stage's points (``gnn.stage_forward``,
   CUDA kernels).
2. The device quantizer codes x against mu, with the reference's exact
   rounding and bound check.
3. log2 b becomes per-point scale levels (``rans.scale_to_level``).
4. The codes are entropy-coded by the native per-point lane coder with the
   dictionary shape of least cost (``rans.choose_shape``).
5. The reconstruction finalises the stage's embeddings before the next stage.

The decoder repeats the same float path and dequantizes on the device.

Scope of this version:

* Tensors above 2^21 points (or with a ``chunk_size``) are cut into a chunk
  grid (the reference's automatic edges); every chunk is an independent
  region with its own anchors (no halo context from its neighbours, unlike
  the reference), and chunks of one shape are coded together as one batch
  through the GNN, the gate, the quantizer and one rANS blob per stage.
* The scale-gated interpolation fallback (``gate=True``, the default) is
  chosen per stage: the encoder scores the GNN against the cubic,
  first-axis-linear and last-axis-linear interpolation of the stage's points
  with the reference's rANS-aligned Laplace rate, per bucket of the model's
  scale relative to eb * 2^T (``latec/gnn_codec.py:386-462, 920-1000``), and
  keeps the GNN only where it codes fewer bits. One gate word per stage, in
  the reference's bit layout, travels in the header. With ``gate_fine`` the
  finest level's sub-stages share one word per region batch, chosen at the
  first of them (``latec/gnn_codec.py:453-462,1229-1262``); those words travel
  apart from the per-stage ones, as the reference's ``fine_gates``.
* Float, signed and unsigned integer and bool inputs: integers are coded in
  normalised float32; for signed integers and bools the bound is checked on
  the nearest raw integer the decoder returns (``round_output`` with the data
  span and minimum), as in the reference.
* ``fp16=True`` (the default, as in the reference) runs the message and
  finalisation MLPs in BF16 on the tensor cores (tcgen05) with float32
  accumulation; pools and the readout stay float32. ``fp16=False`` is float32
  throughout. ``compile`` is accepted and recorded as not compiled.

``fp8=True`` (an extension) runs those MLPs in FP8 (E4M3) with per-channel
weight and per-row activation scales instead. Streams carry their
``"float_path"`` (``latec_b200-bf16-4``, ``latec_b200-fp8-3`` or
``latec_b200-f32-3``). As the reference's own encoder/decoder contract
requires, they decode only with that float path.
"""

from __future__ import annotations

import hashlib
import json
import struct
from pathlib import Path

import numpy as np

from . import _lib, bitstream, gnn, rans, rans_model
from .levels import stage_ebs, stage_strides

MAGIC = b"LATECGNN"
VERSION = 14
PREFIX = "<8sII"
PREFIX_SIZE = struct.calcsize(PREFIX)
FLOAT_PATHS = {"f32": "latec_b200-f32-3", "bf16": "latec_b200-bf16-4",
               "fp8": "latec_b200-fp8-3"}
AUTO_CHUNK_THRESHOLD = 1 << 21
RANK_LEVELS = {2: 8, 4: 5, 5: 4}
EB_COARSE_FACTOR = 0.9
EB_COARSE_SWEEP = (1.0, 0.9, 0.65, 0.41)
# the predictor ablation (latec/gnn_codec.py:755-774): the model replaced by
# the gate's interpolation candidate of that kind, coded against a flat scale
INTERP_KINDS = {"interp-cubic": 1, "interp-linear": 2, "interp-linear-last": 3}
# gate sweep (latec/gnn_codec.py:399-403): thresholds eb * 2^T, scale shifts,
# and the word layout dir (bit 10) | kind (bits 8-9) | T (bits 4-7) | shift
GATE_T = tuple(range(2, 14))
GATE_SHIFTS = (0, 2, 4, 6)
GATE_DIR_SHIFT = 10
GATE_END_MODE = 3  # quadratic ends and extrapolation past the line end
# candidate k: (order, center) of the interpolation predictor
GATE_KINDS = {1: (1, 0), 2: (0, 1), 3: (0, 2)}
_GATE_GRIDS: dict = {}


def _torch():
    import torch

    return torch


def auto_levels(shape, agg_level=2):
    """``latec/gnn_codec.py:69-95``: schedule depth from the input rank,
    capped so the anchor stride stays <= half the largest axis."""
    ndim = len(shape)
    if ndim == 3:
        rank_levels = 7 if agg_level == 1 else 6
    elif ndim in RANK_LEVELS:
        rank_levels = RANK_LEVELS[ndim]
    else:
        rank_levels = (AUTO_CHUNK_THRESHOLD.bit_length() - 1) // ndim
    size_cap = max(1, (int(max(shape)).bit_length() - 1) - 1)
    return max(1, min(rank_levels, size_cap))


def per_step_eb_ratio(coarse_factor, levels):
    """``latec/gnn_codec.py:111-122``."""
    if levels <= 1:
        return 1.0
    return float(coarse_factor) ** (1.0 / (levels - 1))


def write_stream(meta, payload: bytes, zstd_level: int) -> bytes:
    header = json.dumps(meta, sort_keys=True, separators=(",", ":")).encode("utf-8")
    body = bitstream.zstd().compress(np.frombuffer(payload, np.uint8), int(zstd_level))
    return struct.pack(PREFIX, MAGIC, VERSION, len(header)) + header + body


def read_stream(stream: bytes):
    if len(stream) < PREFIX_SIZE:
        raise ValueError("not a LATEC GNN stream")
    magic, version, hlen = struct.unpack_from(PREFIX, stream, 0)
    if magic != MAGIC:
        raise ValueError(f"not a LATEC GNN stream (bad magic {magic!r})")
    if version != VERSION:
        raise ValueError(f"unsupported LATEC GNN stream version {version}")
    if PREFIX_SIZE + hlen > len(stream):
        raise ValueError("truncated LATEC GNN stream header")
    meta = json.loads(stream[PREFIX_SIZE:PREFIX_SIZE + hlen].decode("utf-8"))
    payload = bitstream.zstd().decompress_into(
        np.frombuffer(stream[PREFIX_SIZE + hlen:], np.uint8)).tobytes()
    return meta, payload


def _qparams(radius, raw_round=None):
    """Quantizer parameters; ``raw_round = (span, offset)`` checks the bound
    on the nearest raw integer of integer sources (``_quantize_t``'s
    ``round_output`` pair, latec/gnn_codec.py:998-1031)."""
    if raw_round:
        return _lib.QuantParams(dtype=_lib.F32, channels=1, radius=int(radius), order=1, center=0,
                                end_mode=1, round_output=2, reserved=0,
                                round_span=float(raw_round[0]), round_offset=float(raw_round[1]))
    return _lib.QuantParams(dtype=_lib.F32, channels=1, radius=int(radius), order=1, center=0,
                            end_mode=1, round_output=0, reserved=0)


def _restore_dtype(out, dtype):
    """Decoded float32 values back to the source dtype: integers round to the
    nearest and clip to the type's range, bools threshold at 0.5
    (latec/gnn_codec.py:179-185)."""
    torch = _torch()
    if dtype.kind in "iu":
        info = np.iinfo(dtype)
        r = torch.clamp(torch.round(out.double()), float(info.min), float(info.max))
        return r.to(getattr(torch, dtype.name))
    if dtype.kind == "b":
        return out >= 0.5
    return out.to(getattr(torch, dtype.name)) if dtype != np.float32 else out


def auto_chunk_edges(shape, stride):
    """Largest near-isotropic chunk under the automatic point budget
    (``_auto_chunk_edges``, latec/gnn_codec.py:286-314): axes shorter than the
    budget's edge are taken whole; edges are multiples of the anchor stride."""
    target = AUTO_CHUNK_THRESHOLD
    fixed, remaining = 1, len(shape)
    full = set()
    for axis in sorted(range(len(shape)), key=lambda a: shape[a]):
        free_edge = (target / fixed) ** (1.0 / remaining)
        if shape[axis] > free_edge:
            break
        full.add(axis)
        fixed *= shape[axis]
        remaining -= 1
        if not remaining:
            break
    free_edge = (target / fixed) ** (1.0 / remaining) if remaining else 0.0
    return tuple(max(stride, -(-n // stride) * stride) if a in full
                 else max(stride, int(free_edge) // stride * stride)
                 for a, n in enumerate(shape))


def chunk_edges(shape, stride, chunk_size):
    """Chunk edges, or None when the tensor is coded as one region: ``None``
    chunk_size chunks only tensors above the automatic budget
    (``_chunk_edges``, latec/gnn_codec.py:1549-1574)."""
    if chunk_size is None:
        if int(np.prod(shape)) <= AUTO_CHUNK_THRESHOLD:
            return None
        edges = auto_chunk_edges(shape, stride)
    else:
        edges = ((int(chunk_size),) * len(shape) if np.isscalar(chunk_size)
                 else tuple(int(e) for e in chunk_size))
        if len(edges) != len(shape):
            raise ValueError("chunk_size must be scalar or one entry per axis")
        for e in edges:
            if e < stride or e % stride:
                raise ValueError("chunk_size must be a positive multiple of anchor_stride")
    return None if all(e >= n for e, n in zip(edges, shape)) else tuple(edges)


def chunk_groups(shape, edges):
    """Chunks of the grid in raster order, grouped by their shape (groups in
    order of first appearance): [(chunk shape, [origins])]."""
    grid = [-(-n // e) for n, e in zip(shape, edges)]
    groups = {}
    for idx in np.ndindex(*grid):
        origin = tuple(i * e for i, e in zip(idx, edges))
        cshape = tuple(min(e, n - o) for e, n, o in zip(edges, shape, origin))
        groups.setdefault(cshape, []).append(origin)
    return list(groups.items())


def _chunk_slices(origin, cshape):
    return tuple(slice(o, o + c) for o, c in zip(origin, cshape))


def gate_scale_grid(eb: float, device):
    """The gate's 64-level log scale grid for bound eb (``_gate_scale_thresholds``,
    latec/gnn_codec.py:876-917): float32 level boundaries found by bisection
    over positive float32 bit patterns, and the float64 grid values."""
    import numpy as _np

    torch = _torch()
    key = (str(device), float(eb))
    hit = _GATE_GRIDS.get(key)
    if hit is not None:
        return hit
    from .rans_model import SCALE_HI_MULT, SCALE_LO_DIV

    lo_f, hi_f = float(eb) / SCALE_LO_DIV, float(eb) * SCALE_HI_MULT
    log_lo = _np.log(lo_f)
    log_step = (_np.log(hi_f) - log_lo) / 63.0
    targets = _np.arange(1, 64)
    lo = _np.zeros(63, _np.uint32)
    hi = _np.full(63, _np.asarray(_np.float32(hi_f)).view(_np.uint32), _np.uint32)
    while _np.any(lo < hi):
        mid = lo + (hi - lo) // 2
        v = mid.view(_np.float32).astype(_np.float64)
        level = _np.rint((_np.log(_np.clip(v, lo_f, hi_f)) - log_lo) / log_step)
        up = level >= targets
        hi = _np.where(up, mid, hi).astype(_np.uint32)
        lo = _np.where(up, lo, mid + 1).astype(_np.uint32)
    thr = torch.from_numpy(_np.ascontiguousarray(lo.view(_np.float32))).to(device)
    grid = torch.from_numpy(_np.exp(log_lo + log_step * _np.arange(64))).to(device)
    _GATE_GRIDS[key] = (thr, grid)
    return thr, grid


def gate_choose(sums) -> tuple[int, int, int, int]:
    """(kind, dir, T, shift) from the per-bucket rate sums (rows: GNN, then
    candidate k x shift; columns: scale buckets), the split rule of
    ``_gate_select_t`` (latec/gnn_codec.py:920-971): a low-side split falls
    back where b < eb 2^T, a high-side split where b >= eb 2^T; kind 0 = the
    GNN everywhere (no split codes fewer bits)."""
    W = np.asarray(sums, np.float64).reshape(1 + 3 * len(GATE_SHIFTS), len(GATE_T) + 1)
    cums = np.cumsum(W, axis=1)
    base = cums[0]
    tot = base[-1]
    ci = cums[1:]
    low = tot - base[:-1] + ci[:, :-1]
    high = base[:-1] + (ci[:, -1:] - ci[:, :-1])
    costs = np.concatenate([low, high]).reshape(-1)
    fi = int(np.argmin(costs))
    if not costs[fi] < tot:
        return 0, 0, 0, 0
    ncol, nsh = len(GATE_T), len(GATE_SHIFTS)
    n_side = 3 * nsh
    row = fi // ncol
    side_row = row % n_side
    return side_row // nsh + 1, int(row >= n_side), GATE_T[fi % ncol], GATE_SHIFTS[side_row % nsh]


def gate_word(kind, direction, T, shift) -> int:
    return (int(direction) << GATE_DIR_SHIFT) | (int(kind) << 8) | (int(T) << 4) | int(shift)


def gate_fields(word: int) -> tuple[int, int, int, int]:
    return (word >> 8) & 3, (word >> GATE_DIR_SHIFT) & 1, (word >> 4) & 15, word & 15


def pack_gates(words) -> str:
    """Gate words as base64 of little-endian uint16 (``_pack_gates``)."""
    import base64

    return base64.b64encode(np.asarray(words, "<u2").tobytes()).decode("ascii")


def unpack_gates(blob: str) -> list:
    import base64

    return np.frombuffer(base64.b64decode(blob), "<u2").astype(np.int64).tolist()


class GNNCodec:
    """The learned codec (``latec/gnn_codec.py:1509-1922``)."""

    def __init__(self, checkpoint_path=None, device=None, *, strict_checkpoint=True,
                 weights=None, d=64, agg_level=1):
        """``checkpoint_path``: a v7 axial-GNN checkpoint (as the reference).
        Alternatively ``weights`` (a dict with the reference parameter names,
        e.g. ``gnn.random_weights``) with ``d`` / ``agg_level``."""
        torch = _torch()
        _lib.load()
        if weights is None:
            if checkpoint_path is None:
                raise ValueError("a checkpoint path or a weights dict is required")
            path = Path(checkpoint_path)
            if not path.exists():
                raise FileNotFoundError(f"GNN checkpoint not found: {path}")
            weights, d, agg_level = gnn.load_checkpoint(path)
            h = hashlib.sha256()
            with open(path, "rb") as f:
                for block in iter(lambda: f.read(1 << 20), b""):
                    h.update(block)
            self.checkpoint_hash = h.digest()[:16]
        else:
            h = hashlib.sha256()
            for k in gnn.param_shapes(d, agg_level):
                h.update(np.ascontiguousarray(weights[k], np.float32).tobytes())
            self.checkpoint_hash = h.digest()[:16]
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.strict_checkpoint = bool(strict_checkpoint)
        self.d, self.agg_level = int(d), int(agg_level)
        self._weights = weights
        self._models = {}
        self._geoms = {}
        # a list to receive per-stage device tensors of every encode (model mu
        # and scale, gate word, codes, scale levels, outliers), or None. A
        # test and diagnosis aid: parity checks against the reference codec
        # compare them stage by stage.
        self.stage_trace = None

    def _model(self, precision: str):
        """The model in one float path: "f32", "bf16" (the tensor-core message
        pass, counterpart of the reference's fp16 one) or "fp8" (E4M3 with
        per-channel weight and per-row activation scales); d = 64 for the
        tensor-core paths."""
        m = self._models.get(precision)
        if m is None:
            m = gnn.GNNModel(self._weights, self.d, self.agg_level, self.device,
                             precision=precision)
            self._models[precision] = m
        return m

    # ---------------------------------------------------------------- helpers
    def _geometry(self, shape, levels):
        key = (tuple(shape), int(levels))
        g = self._geoms.get(key)
        if g is None:
            stride = 1 << int(levels)
            g = gnn.build_stage_geoms(shape, levels, stride, 1, stride, self.agg_level,
                                      device=self.device)[0]
            self._geoms = {key: g}  # one shape at a time
        return g

    def _stage_ebs(self, shape, levels, eb, ratio):
        """Per non-empty stage eb, in the geometry's stage order."""
        from .levels import plan_for

        stride = 1 << int(levels)
        ebs = stage_ebs(shape, levels, stride, 1, eb, ratio)
        counts = plan_for(shape, levels, stride, 1).counts
        return [float(e) for e, n in zip(ebs, counts) if n]

    # ---------------------------------------------------------------- encode
    def compress(self, x, error_bound: float = 1e-2, *, levels="auto", radius: int = 1 << 15,
                 zstd_level: int = 9, eb_ratio=None, tune: str = "fast", chunk_size=None,
                 fp16: bool = True, compile="auto", gate: bool = True, gate_fine: bool = False,
                 predictor: str = "gnn", fp8: bool = False) -> bytes:
        """Compress a NumPy array or torch tensor (``latec/gnn_codec.py:1576-1775``).
        ``fp8=True`` (no counterpart in the reference) runs the message-pass
        MLPs in FP8 instead of BF16; the stream records that float path."""
        torch = _torch()
        if tune not in ("fast", "size"):
            raise ValueError("tune must be 'fast' or 'size'")
        if isinstance(levels, str) and levels != "auto":
            raise ValueError("levels must be a positive int or 'auto'")
        if isinstance(compile, str) and compile != "auto":
            raise ValueError("compile must be a bool or 'auto'")
        if not isinstance(levels, str) and int(levels) < 1:
            raise ValueError("levels must be >= 1")
        if predictor != "gnn" and predictor not in INTERP_KINDS:
            raise ValueError(f"predictor must be 'gnn' or one of {sorted(INTERP_KINDS)}")
        interp_kind = INTERP_KINDS.get(predictor, 0)
        radius = int(radius)
        if not 1 <= radius <= 32768:
            raise ValueError("radius must be in [1, 32768]")
        gate = bool(gate) and not interp_kind  # no model prediction to fall back from
        gate_fine = bool(gate_fine) and gate
        is_t = isinstance(x, torch.Tensor)
        arr = x.detach() if is_t else np.asarray(x)
        if (arr.numel() if is_t else arr.size) == 0:
            raise ValueError("cannot compress an empty tensor")
        np_dtype = np.dtype(str(arr.dtype).replace("torch.", "")) if is_t else np.dtype(arr.dtype)
        if np_dtype.kind not in "biuf":
            raise TypeError(f"unsupported dtype {np_dtype}; expected numeric data")
        eb = float(error_bound)
        if eb <= 0:
            raise ValueError("error_bound must be > 0")
        original_shape = tuple(int(n) for n in arr.shape)
        shape = original_shape if original_shape else (1,)
        lv = auto_levels(shape, self.agg_level) if isinstance(levels, str) else int(levels)
        stride = 1 << lv
        cedges = chunk_edges(shape, stride, chunk_size)
        edges = cedges or tuple(-(-n // stride) * stride for n in shape)
        t = arr if is_t else torch.from_numpy(np.ascontiguousarray(arr))
        t = t.reshape(shape).to(self.device)
        if np_dtype.kind != "f":  # integer / bool sources are coded in float32
            t = t.to(torch.float32)
        mm = torch.aminmax(t)
        vmin = float(np.float32(float(mm.min.item())))
        vmax = float(np.float32(float(mm.max.item())))
        if vmax <= vmin:
            vmax = vmin + 1.0
        span = vmax - vmin
        xn = ((t.to(torch.float32) - np.float32(vmin)) / np.float32(span)).reshape(-1).contiguous()
        # signed integers and bools are finally rounded to the nearest raw
        # integer, so the bound is checked on that value
        raw_round = (span, vmin) if np_dtype.kind in "bi" else None
        coarse = ([float(eb_ratio)] if eb_ratio is not None
                  else (list(EB_COARSE_SWEEP) if tune == "size" else [EB_COARSE_FACTOR]))
        ratios = sorted({per_step_eb_ratio(c, lv) for c in coarse})
        best = None
        reduced = bool(fp16) and self.d == 64
        precision = ("fp8" if fp8 else "bf16") if reduced else "f32"
        if fp8 and not reduced:
            raise ValueError("fp8 needs the tensor-core path (fp16=True, d = 64)")
        model = self._model(precision)
        cbatch = self._chunk_batch(edges) if cedges else 1
        for ratio in ratios:
            if cedges is None:
                payload, words, fine_words = self._encode(model, xn.reshape(1, -1), shape, lv,
                                                          eb, ratio, radius, gate, raw_round,
                                                          gate_fine, interp_kind)
            else:  # chunks of one shape coded in batches
                xg = xn.reshape(shape)
                parts, words, fine_words = [], [], []
                for cshape, origins in chunk_groups(shape, edges):
                    for b0 in range(0, len(origins), cbatch):
                        X = torch.stack([xg[_chunk_slices(o, cshape)].reshape(-1)
                                         for o in origins[b0:b0 + cbatch]])
                        part, w, fw = self._encode(model, X, cshape, lv, eb, ratio, radius,
                                                   gate, raw_round, gate_fine, interp_kind)
                        parts.append(part)
                        words += w
                        fine_words += fw
                payload = b"".join(parts)
            meta = {"shape": list(original_shape), "dtype": np_dtype.str, "error_bound": eb,
                    "levels": lv, "radius": radius, "vmin": vmin, "vmax": vmax,
                    "eb_ratio": ratio, "checkpoint_hash": self.checkpoint_hash.hex(),
                    "chunks": list(edges), "m_tile": 1 << 16, "fp16": reduced, "compiled": False,
                    "predictor": predictor, "float_path": FLOAT_PATHS[precision], "d": self.d,
                    "agg_level": self.agg_level, "gate": gate, "gate_fine": gate_fine,
                    "gates": pack_gates(words)}
            if gate_fine:
                meta["fine_gates"] = pack_gates(fine_words)
            if cedges is not None:
                meta["chunk_batch"] = cbatch
            if int(model.tc_err.item()):
                raise RuntimeError("a tensor-core wait ran out during the GNN forward")
            stream = write_stream(meta, payload, zstd_level)
            if best is None or len(stream) < len(best):
                best = stream
        return best

    def _plan_stages(self, shape, levels):
        """The interpolation plan of the schedule and its stage index per
        non-empty GNN stage."""
        from .levels import plan_for

        plan = plan_for(shape, levels, 1 << levels, 1)
        return plan, [t for t, n in enumerate(plan.counts) if n]

    def _chunk_batch(self, edges):
        """Chunks coded together: the embedding field of a batch (chunk points
        x axes x d float32) and its message-pass workspace stay near 16 GB."""
        per = int(np.prod(edges)) * len(edges) * self.d * 4 * 3
        return max(1, min(64, int(16e9 // per)))

    def _gate_candidate(self, plan, stage, kind, recon_all, n, radius):
        """Interpolation candidate ``kind`` (1 cubic axis-average, 2 first-axis
        linear, 3 last-axis linear) of a stage from the reconstruction
        ``recon_all`` (B, N): n = B * stage points, region-major."""
        import ctypes

        torch = _torch()
        order, center = GATE_KINDS[kind]
        out = torch.empty(n, dtype=torch.float32, device=self.device)
        prm = _lib.QuantParams(dtype=_lib.F32, channels=int(recon_all.shape[0]),
                               radius=int(radius), order=order,
                               center=center, end_mode=GATE_END_MODE, round_output=0, reserved=0)
        _lib.check(_lib.load().latec_interp_predict_stage(plan.handle, stage, ctypes.byref(prm),
                                                          recon_all.data_ptr(), out.data_ptr(),
                                                          _lib.stream_ptr()),
                   "latec_interp_predict_stage")
        return out

    def _interp_stage(self, plan, stage, gi, kind, recon_all, n, seb, radius):
        """(prediction, scale) of a stage under the interpolation ablation
        (``_interp_stage_pred``, latec/gnn_codec.py:763-774): the gate's
        candidate of ``kind`` (0 for the anchors, as the reference's anchor
        pass) and a flat scale of the stage's eb."""
        torch = _torch()
        mu = (self._gate_candidate(plan, stage, kind, recon_all, n, radius) if gi else
              torch.zeros(n, dtype=torch.float32, device=self.device))
        return mu, torch.full((n,), float(seb), dtype=torch.float32, device=self.device)

    def _encode(self, model, X, shape, levels, eb, ratio, radius, gate=True, raw_round=None,
                gate_fine=False, interp_kind=0):
        """Code B regions of one shape at once: X (B, N) normalised values.
        Every stage runs the GNN over the batch, and its codes (region-major)
        form one rANS blob; one gate word per stage serves the batch. With
        ``gate_fine`` the finest level's sub-stages reuse the gate chosen at
        the first of them. ``interp_kind`` codes with that interpolation
        candidate instead of the model, against a flat scale of the stage's eb
        (the anchors against 0). Returns (payload, per-stage words, finest
        words)."""
        torch = _torch()
        lib = _lib.load()
        geoms = self._geometry(shape, levels)
        ebs = self._stage_ebs(shape, levels, eb, ratio)
        plan, pstages = self._plan_stages(shape, levels)
        prm = _qparams(radius, raw_round)
        dev = self.device
        B, N = int(X.shape[0]), int(X.shape[1])
        E = None if interp_kind else torch.zeros((B, N, len(shape), self.d),
                                                 dtype=torch.float32, device=dev)
        recon_all = torch.zeros((B, N), dtype=torch.float32, device=dev)
        strides = stage_strides(len(shape), levels, 1 << levels)
        finest = [strides[t] == 1 for t in pstages]
        # every stage's codes, level rows, outliers and statistics stay on the
        # device until the entropy step after the stage loop
        offs = np.concatenate([[0], np.cumsum([B * g.M for g in geoms])]).astype(np.int64)
        total = max(int(offs[-1]), 1)
        codes_all = torch.empty(total, dtype=torch.int16, device=dev)
        lv_all = torch.empty(total, dtype=torch.uint8, device=dev)
        outl_all = torch.empty(total, dtype=torch.float32, device=dev)
        ssz = ctypes_sizeof_stats()
        stats_all = torch.zeros(max(len(geoms), 1) * ssz, dtype=torch.uint8, device=dev)
        # gate words, chosen on the device and read once the batch is coded
        gw = torch.zeros(max(len(geoms), 1), dtype=torch.int32, device=dev)
        fine_gi = None
        prev, ctx, vals = None, None, None
        for gi, (g, seb) in enumerate(zip(geoms, ebs)):
            n = B * g.M
            if gi == 0 or interp_kind:
                # the anchor stage is coded against 0 with a flat scale of its
                # eb, before the model runs (latec/gnn_codec.py:358-373); the
                # first model stage embeds the anchors from their reconstruction
                mu, scale = self._interp_stage(plan, pstages[gi], gi, interp_kind, recon_all, n,
                                               seb, radius)
            else:
                (mu, lb), E, ctx = gnn.stage_forward(model, E, prev, g, vals, finalize_ctx=ctx,
                                                     eb=seb)
                mu = mu.reshape(-1).contiguous()
                scale = torch.exp2(lb.reshape(-1)).contiguous()
            xs = X[:, g.query_idx].reshape(-1).contiguous()
            if self.stage_trace is not None:
                tr = {"stage": gi, "eb": seb, "mu": mu.clone(), "scale": scale.clone(),
                      "x": xs.clone()}
            shared = gate_fine and finest[gi]
            if gate and gi > 0 and n:
                # the interpolation fallback, scored, chosen (gate_choose's rule)
                # and applied on the device: no host round trip per stage
                ips = [self._gate_candidate(plan, pstages[gi], k, recon_all, n, radius)
                       for k in (1, 2, 3)]
                if shared and fine_gi is not None:
                    _lib.check(lib.latec_gate_apply_word(
                        n, mu.data_ptr(), scale.data_ptr(), ips[0].data_ptr(), ips[1].data_ptr(),
                        ips[2].data_ptr(), seb, gw.data_ptr() + 4 * fine_gi, _lib.stream_ptr()),
                        "latec_gate_apply_word")
                else:
                    sums = torch.zeros(len(GATE_KINDS) * len(GATE_SHIFTS) * (len(GATE_T) + 1)
                                       + len(GATE_T) + 1, dtype=torch.int64, device=dev)
                    thr, grid = gate_scale_grid(seb, dev)
                    _lib.check(lib.latec_gate_costs(n, xs.data_ptr(), mu.data_ptr(),
                                                    ips[0].data_ptr(), ips[1].data_ptr(),
                                                    ips[2].data_ptr(), scale.data_ptr(), seb,
                                                    radius, thr.data_ptr(), grid.data_ptr(),
                                                    sums.data_ptr(), _lib.stream_ptr()),
                               "latec_gate_costs")
                    _lib.check(lib.latec_gate_choose_apply(
                        n, sums.data_ptr(), mu.data_ptr(), scale.data_ptr(), ips[0].data_ptr(),
                        ips[1].data_ptr(), ips[2].data_ptr(), seb, gw.data_ptr() + 4 * gi,
                        _lib.stream_ptr()), "latec_gate_choose_apply")
                    if shared:
                        fine_gi = gi
            o = int(offs[gi])
            recon = torch.empty(n, dtype=torch.float32, device=dev)
            hseg = torch.empty(max(1, -(-n // (1 << 22))) * 512, dtype=torch.int32, device=dev)
            htot = torch.empty(65536, dtype=torch.int32, device=dev)
            ws = torch.empty(int(lib.latec_flat_workspace_bytes(n, _lib.F32)), dtype=torch.uint8,
                             device=dev)
            _lib.check(lib.latec_quantize(_byref(prm), seb, n, xs.data_ptr(), mu.data_ptr(),
                                          codes_all.data_ptr() + 2 * o, recon.data_ptr(),
                                          outl_all.data_ptr() + 4 * o,
                                          stats_all.data_ptr() + gi * ssz, hseg.data_ptr(),
                                          htot.data_ptr(), ws.data_ptr(), ws.numel(),
                                          _lib.stream_ptr()), "latec_quantize")
            lv_all[o:o + n].copy_(rans.scale_to_level(scale, seb))
            if self.stage_trace is not None:
                tr.update(codes=codes_all[o:o + n].clone(), levels=lv_all[o:o + n].clone(),
                          mu_gated=mu.clone(), scale_gated=scale.clone(),
                          word=gw[fine_gi if shared and fine_gi is not None else gi].clone(),
                          recon=recon.clone(), outliers=outl_all[o:o + n].clone())
                self.stage_trace.append(tr)
            recon_all[:, g.query_idx] = recon.reshape(B, -1)
            prev, vals = g, recon.reshape(B, -1)
        payload = self._entropy(ebs, offs, codes_all, lv_all, outl_all, stats_all, radius)
        got = gw.cpu().numpy().astype(np.int64).tolist()
        words = [got[gi] for gi in range(len(geoms)) if not (gate_fine and finest[gi])]
        fine_words = [got[fine_gi]] if fine_gi is not None else []
        return payload, words, fine_words

    def _entropy(self, ebs, offs, codes_all, lv_all, outl_all, stats_all, radius):
        """The stage records of one batch (``u32 n | u64 frame | blob | u32
        n_out | outliers``, the per-point native rANS of ``latec_b200.rans``
        for every stage): per stage the coder window from the largest code and
        the table shape of least cost, then every stage through the lane coder
        and the record assembly in one launch."""
        torch = _torch()
        lib = _lib.load()
        dev = self.device
        ns = len(ebs)
        if ns == 0:
            return b""
        ssz = ctypes_sizeof_stats()
        raw = stats_all.cpu().numpy().tobytes()  # one download: every stage's statistics
        st = (_lib.StageStats * ns).from_buffer_copy(raw[:ns * ssz])
        kexps = [max(1, int(st[t].maxq).bit_length()) for t in range(ns)]
        tabs = [rans.build_laplace_tables(seb, radius) for seb in ebs]
        costs = [rans.shape_costs(codes_all.data_ptr() + 2 * int(offs[t]),
                                  lv_all.data_ptr() + int(offs[t]), int(offs[t + 1] - offs[t]),
                                  tabs[t], kexps[t], dev) for t in range(ns)]
        got = torch.cat([c[1] for c in costs]).cpu().numpy()  # one download: shape costs
        shapes, at = [], 0
        for ids, part in costs:
            shapes.append(rans.pick_shape(ids, got[at:at + part.numel()]))
            at += part.numel()
        stages = (_lib.RansStage * ns)()
        keep = []
        for t in range(ns):
            n = int(offs[t + 1] - offs[t])
            cdf, enc, bucket, alphabet = rans_model.device_tables.get(
                _lib.RANS_LANES, kexps[t], shapes[t], 0, None, dev)
            keep.append((cdf, enc, bucket))
            d = stages[t]
            d.codes_off = d.out_off = int(offs[t])
            d.n = n
            d.kexp, d.radius, d.mode, d.per_point = kexps[t], int(radius), _lib.RANS_LANES, 1
            d.alphabet = alphabet
            d.framed_hi = bitstream.pack_frame(0, kexps[t], shapes[t], 0, 0, False)
            d.cdf, d.enc, d.bucket = cdf.data_ptr(), enc.data_ptr(), bucket.data_ptr()
            d.K = rans_model.lanes_K(n, 4.0 * n)
        wsb = lib.latec_rans_encode_workspace_bytes(stages, ns)
        ws = torch.empty(max(int(wsb), 1), dtype=torch.uint8, device=dev)
        cap = sum(16 + 4 * (1 + 65 * int(stages[t].n_chunks) + int(stages[t].n) + 2)
                  + 4 * int(stages[t].n) for t in range(ns))
        cap = (cap + 15) // 16 * 16
        payload = torch.empty(cap, dtype=torch.uint8, device=dev)
        plen = torch.zeros(1, dtype=torch.int64, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        _lib.check(lib.latec_rans_encode(stages, ns, codes_all.data_ptr(), lv_all.data_ptr(),
                                         stats_all.data_ptr(), outl_all.data_ptr(), 4,
                                         payload.data_ptr(), cap, plen.data_ptr(), err.data_ptr(),
                                         ws.data_ptr(), ws.numel(), _lib.stream_ptr()),
                   "latec_rans_encode")
        tail = torch.cat([plen.view(torch.uint8), err.view(torch.uint8)]).cpu().numpy()
        if int(tail[8:12].view(np.int32)[0]):
            raise RuntimeError(f"entropy coder reported error bits "
                               f"{int(tail[8:12].view(np.int32)[0]):#x}")
        n_bytes = int(tail[:8].view(np.int64)[0])
        out = payload[:n_bytes].cpu().numpy().tobytes()
        del keep
        return out

    # ---------------------------------------------------------------- decode
    def uncompress(self, stream):
        """Decompress a stream from ``compress`` into a torch tensor of the
        original shape and dtype (``latec/gnn_codec.py:1777-1830``)."""
        torch = _torch()
        lib = _lib.load()
        meta, payload = read_stream(bytes(stream))
        paths = {v: k for k, v in FLOAT_PATHS.items()}
        if meta.get("float_path") not in paths:
            raise ValueError("stream was not written by this codec's float path")
        model = self._model(paths[meta["float_path"]])
        if self.strict_checkpoint and meta["checkpoint_hash"] != self.checkpoint_hash.hex():
            raise ValueError("checkpoint hash differs from the stream metadata")
        original_shape = tuple(int(n) for n in meta["shape"])
        shape = original_shape or (1,)
        dtype = np.dtype(meta["dtype"])
        vmin, vmax = float(meta["vmin"]), float(meta["vmax"])
        if vmax <= vmin:
            vmax = vmin + 1.0
        levels, radius = int(meta["levels"]), int(meta["radius"])
        eb, ratio = float(meta["error_bound"]), float(meta["eb_ratio"])
        words = unpack_gates(meta["gates"]) if meta.get("gates") else None
        predictor = meta.get("predictor", "gnn")
        if predictor != "gnn" and predictor not in INTERP_KINDS:
            raise ValueError(f"unknown predictor {predictor!r} in stream")
        interp_kind = INTERP_KINDS.get(predictor, 0)
        fine = unpack_gates(meta.get("fine_gates", "")) if meta.get("gate_fine") else None
        if fine is not None and words is None:
            raise ValueError("finest-level gate words without per-stage gate words")
        # error words: [0] the dequantizer, [1] the lane decoder; read once at the end
        err = torch.zeros(2, dtype=torch.int32, device=self.device)
        pay_dev = torch.from_numpy(np.frombuffer(payload + bytes(8), np.uint8).copy()).to(
            self.device)  # the whole payload once; stage blobs and outliers are read in place
        if "chunk_batch" in meta:  # chunks of one shape, decoded in the encoder's batches
            edges = tuple(int(e) for e in meta["chunks"])
            cbatch = int(meta["chunk_batch"])
            if len(edges) != len(shape) or cbatch < 1:
                raise ValueError("malformed chunk grid")
            out = torch.empty(shape, dtype=torch.float32, device=self.device)
            off, wi, fi = 0, 0, 0
            for cshape, origins in chunk_groups(shape, edges):
                for b0 in range(0, len(origins), cbatch):
                    sub = origins[b0:b0 + cbatch]
                    R, off, wi, fi = self._decode(model, payload, pay_dev, off, len(sub),
                                                  cshape, levels, eb, ratio, radius, words, wi,
                                                  fine, fi, err, interp_kind)
                    for j, o in enumerate(sub):
                        out[_chunk_slices(o, cshape)] = R[j].reshape(cshape)
            recon_all = out.reshape(-1)
        else:
            R, off, wi, fi = self._decode(model, payload, pay_dev, 0, 1, shape, levels, eb,
                                          ratio, radius, words, 0, fine, 0, err, interp_kind)
            recon_all = R.reshape(-1)
        if off != len(payload):
            raise ValueError("trailing data in GNN stage payload")
        if (words is not None and wi != len(words)) or (fine is not None and fi != len(fine)):
            raise ValueError("gate words do not match the stage schedule")
        e_dq, e_rans = (int(v) for v in err.cpu().tolist())
        if e_rans & (4 | 8):
            raise ValueError("trailing data in rANS payload")
        if e_rans:
            raise ValueError(f"malformed rANS payload (error bits {e_rans:#x})")
        if e_dq:
            raise ValueError("outlier count mismatch")
        if int(model.tc_err.item()):
            raise RuntimeError("a tensor-core wait ran out during the GNN forward")
        out = recon_all * np.float32(vmax - vmin) + np.float32(vmin)
        return _restore_dtype(out.reshape(original_shape).cpu(), dtype)

    def _decode(self, model, payload, pay_dev, off, B, shape, levels, eb, ratio, radius, words,
                wi, fine, fi, err, interp_kind=0):
        """Decode B regions of one shape from ``payload`` (host bytes; its
        device copy ``pay_dev``) at ``off``, reading per-stage gate words from
        ``words[wi:]`` and, when the stream shares one word over the finest
        level, that word from ``fine[fi]``; returns (recon (B, N), the offset
        after them, the next wi, the next fi). The stage records are parsed on
        the host first; each stage's codes are then rANS-decoded on the device
        from the payload copy and dequantized there, and the error words
        ``err`` are read by the caller."""
        torch = _torch()
        lib = _lib.load()
        geoms = self._geometry(shape, levels)
        ebs = self._stage_ebs(shape, levels, eb, ratio)
        prm = _qparams(radius)
        dev = self.device
        N = int(np.prod(shape))
        recon_all = torch.zeros((B, N), dtype=torch.float32, device=dev)
        E = None if interp_kind else torch.zeros((B, N, len(shape), self.d),
                                                 dtype=torch.float32, device=dev)
        prev, ctx, vals = None, None, None
        plan, pstages = self._plan_stages(shape, levels)
        strides = stage_strides(len(shape), levels, 1 << levels)
        shared = [fine is not None and strides[t] == 1 for t in pstages]
        if words is not None and wi + shared.count(False) > len(words):
            raise ValueError("gate words do not match the stage schedule")
        if any(shared) and fi >= len(fine):
            raise ValueError("gate words do not match the stage schedule")
        recs = []  # per stage: (n, frame fields, blob byte offset, outliers byte offset, n_out)
        chunk_ranges = []
        for g in geoms:
            if off + 12 > len(payload):
                raise ValueError("truncated GNN stage payload")
            n, frame = struct.unpack_from("<IQ", payload, off)
            f = bitstream.unpack_frame(frame)
            if n != B * g.M:
                raise ValueError("stage size differs from the schedule")
            if f["hlen"] % 4:
                raise ValueError("rANS payload is not aligned to 32-bit words")
            bo = off + 12
            off = bo + f["hlen"]
            if off + 4 > len(payload):
                raise ValueError("truncated GNN stage payload")
            (n_out,) = struct.unpack_from("<I", payload, off)
            off += 4
            if n_out > n or off + 4 * n_out > len(payload):
                raise ValueError("truncated GNN stage payload")
            # the lane coder's chunk table: K, then each chunk's word count
            wd = np.frombuffer(payload, "<u4", count=f["hlen"] // 4, offset=bo)
            if len(wd) < 1 or int(wd[0]) < 1:
                raise ValueError("malformed rANS payload")
            K = int(wd[0])
            nc = -(-n // (32 * K))
            if len(wd) < 1 + nc:
                raise ValueError("malformed rANS payload")
            ends = 1 + nc + np.cumsum(wd[1:1 + nc].astype(np.int64))
            if int(ends[-1]) != len(wd):
                raise ValueError("trailing data in rANS payload")
            starts = ends - wd[1:1 + nc].astype(np.int64)
            chunk_ranges.append(np.stack([starts, ends], 1).reshape(-1) + bo // 4)
            recs.append((n, f, bo, off, n_out, K, nc))
            off += 4 * n_out
        ranges = torch.from_numpy(np.concatenate(chunk_ranges)).to(dev)  # one upload
        ch0 = np.concatenate([[0], np.cumsum([r[6] for r in recs])]).astype(np.int64)
        fine_desc = None
        for gi, (g, seb) in enumerate(zip(geoms, ebs)):
            if gi == 0 or interp_kind:  # the anchors: against 0, as the encoder
                mu, scale = self._interp_stage(plan, pstages[gi], gi, interp_kind, recon_all,
                                               B * g.M, seb, radius)
            else:
                (mu, lb), E, ctx = gnn.stage_forward(model, E, prev, g, vals, finalize_ctx=ctx,
                                                     eb=seb)
                mu = mu.reshape(-1).contiguous()
                scale = torch.exp2(lb.reshape(-1)).contiguous()
            n, f, bo, oo, n_out, K, nc = recs[gi]
            if shared[gi]:
                if fine_desc is None:
                    fine_desc = gate_fields(int(fine[fi]))
                    fi += 1
                kind, direction, T, shift = fine_desc
            elif words is not None:
                kind, direction, T, shift = gate_fields(int(words[wi]))
                wi += 1
            else:
                kind, direction, T, shift = 0, 0, 0, 0
            if kind:
                if gi == 0 or kind not in GATE_KINDS:
                    raise ValueError("invalid gate word")
                ip = self._gate_candidate(plan, pstages[gi], kind, recon_all, n, radius)
                _lib.check(lib.latec_gate_apply(n, mu.data_ptr(), scale.data_ptr(), ip.data_ptr(),
                                                seb, T, shift, direction, _lib.stream_ptr()),
                           "latec_gate_apply")
            # the stage's codes: per-point native rANS (latec_b200.rans.rans_decode),
            # decoded on the device from the payload copy
            lv64 = rans.scale_to_level(scale, seb)
            cdf, enc, bucket, alphabet = rans_model.device_tables.get(
                _lib.RANS_LANES, f["kexp"], f["shape"], 0, None, dev)
            st = (_lib.RansStage * 1)()
            d = st[0]
            d.codes_off, d.n = 0, n
            d.kexp, d.radius, d.mode, d.per_point = f["kexp"], int(radius), _lib.RANS_LANES, 1
            d.alphabet = alphabet
            d.cdf, d.enc, d.bucket = cdf.data_ptr(), enc.data_ptr(), bucket.data_ptr()
            d.blob_off, d.blob_words = bo // 4, f["hlen"] // 4
            d.K, d.n_chunks, d.chunk0 = K, nc, 0
            codes_d = torch.empty(n, dtype=torch.int16, device=dev)
            rws = torch.empty(int(lib.latec_rans_decode_workspace_bytes(1)), dtype=torch.uint8,
                              device=dev)
            _lib.check(lib.latec_rans_decode(st, 1, nc, pay_dev.data_ptr(),
                                             ranges.data_ptr() + 16 * int(ch0[gi]),
                                             lv64.data_ptr(), codes_d.data_ptr(),
                                             err.data_ptr() + 4, rws.data_ptr(), rws.numel(),
                                             _lib.stream_ptr()), "latec_rans_decode")
            recon = torch.empty(n, dtype=torch.float32, device=dev)
            ws = torch.empty(max(int(lib.latec_dequantize_workspace_bytes(n)), 1),
                             dtype=torch.uint8, device=dev)
            _lib.check(lib.latec_dequantize(_byref(prm), seb, n, mu.data_ptr(), codes_d.data_ptr(),
                                            pay_dev.data_ptr() + oo, n_out, recon.data_ptr(),
                                            err.data_ptr(), ws.data_ptr(), ws.numel(),
                                            _lib.stream_ptr()), "latec_dequantize")
            del cdf, enc, bucket
            recon_all[:, g.query_idx] = recon.reshape(B, -1)
            prev, vals = g, recon.reshape(B, -1)
        return recon_all, off, wi, fi

    decompress = uncompress


GNNCompressorCodec = GNNCodec


def ctypes_sizeof_stats():
    import ctypes

    return ctypes.sizeof(_lib.StageStats)


def _byref(prm):
    import ctypes

    return ctypes.byref(prm)


