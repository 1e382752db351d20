"""Closed-loop LATEC codec on the GPU: ``compress`` / ``decompress``.

Same public signatures, stream container, per-stage statistics and error
behaviour as the reference driver (``latec/codec.py:45-322``); the stage loop
(``latec/codec.py:384-510``) runs as CUDA kernels through the C ABI:

* encode: one fused predict + quantize + reconstruct kernel per stage writes
  codes, the reconstruction, outliers (compacted in scan order) and the
  stage's symbol histogram; the host fits the stage-constant rANS model from
  the histogram (the reference's float32 fit), then one launch entropy-codes
  every stage and assembles the stage records on the device;
* decode: one launch rANS-decodes every stage's codes, then one predict +
  dequantize kernel per stage rebuilds the field.

Entropy back ends: ``entropy="native"`` (default) writes the 32-lane
interleaved rANS blobs and a raw-block zstd frame (flag ``FLAG_LANES``);
``entropy="compat"`` writes the reference's own single-stack rANS stream,
literal-zstd stages and a level-``zstd_level`` zstd frame, which the
reference's ``decompress`` reads.
"""

from __future__ import annotations

import ctypes
import struct
import time

import numpy as np

from . import _lib, bitstream, levels, rans_model
from .bitstream import (DTYPE_CODES, DTYPE_IDS, END_MODE_SHIFT, FLAG_CUBIC, FLAG_INTERP,
                        FLAG_LANES, FLAG_RANS, Header)

END_MODE_MAX = 3


def _torch():
    import torch

    return torch


def _is_tensor(x):
    try:
        import torch

        return isinstance(x, torch.Tensor)
    except Exception:  # pragma: no cover
        return False


def _np_dtype(x):
    if _is_tensor(x):
        torch = _torch()
        m = {torch.uint8: np.uint8, torch.float32: np.float32, torch.float64: np.float64,
             torch.float16: np.float16, torch.int16: np.int16, torch.int32: np.int32,
             torch.int64: np.int64, torch.bfloat16: None}
        dt = m.get(x.dtype)
        return np.dtype(dt) if dt is not None else None
    return np.dtype(x.dtype)


def _prepare(img, device):
    """Shape normalisation of ``latec/codec.py:72-91`` plus float64; returns the
    channel-first device field and its description."""
    torch = _torch()
    if not _is_tensor(img):
        img = np.asarray(img)
    ndim = img.ndim
    shape = tuple(int(n) for n in img.shape)
    is_image = ndim <= 2 or (ndim == 3 and shape[-1] in (1, 3))
    dt = _np_dtype(img)
    if dt is None or dt not in DTYPE_IDS:
        raise KeyError(dt)
    src = DTYPE_IDS[dt]
    if not is_image:
        spatial, c = shape, 1
    elif ndim == 2:
        spatial, c = shape, 1
    elif ndim == 3:
        spatial, c = shape[:-1], shape[-1]
    else:  # 0-D / 1-D input: the reference's image branch leaves no spatial axis
        spatial, c = shape[:-1], 1
    if len(spatial) < 1:
        raise ValueError("shape must have at least one axis")
    ft = torch.float64 if src == 2 else torch.float32
    t = img if _is_tensor(img) else torch.from_numpy(np.ascontiguousarray(img))
    t = t.to(device=device, non_blocking=True)
    t = t.to(ft)
    if is_image and ndim == 3:
        t = t.movedim(-1, 0)
    else:
        t = t.reshape((1,) + tuple(spatial))
    return t.contiguous(), tuple(spatial), c, src


class _Buffers:
    """Device buffers of one compress/decompress call, reused across tune candidates.
    ``views`` (kind -> tensor of ``sizes()``'s length and dtype) places the
    codes, outliers, stage statistics and histograms in buffers shared with
    other tensors (``latec_b200.batch``)."""

    def __init__(self, plan, c, dtype_id, device, views=None):
        torch = _torch()
        self.torch = torch
        self.plan = plan
        self.c = c
        self.elem = 8 if dtype_id == 2 else 4
        self.ldtype = _lib.F64 if dtype_id == 2 else _lib.F32
        self.device = device
        self.items = [n * c for n in plan.counts]
        self.offsets = np.concatenate([[0], np.cumsum(self.items)]).astype(np.int64)
        self.total = int(self.offsets[-1])
        self.segs = [-(-n // rans_model.SEG) for n in self.items]
        self.seg_off = np.concatenate([[0], np.cumsum(self.segs)]).astype(np.int64)
        if views is None:
            views = {k: torch.empty(n, dtype=dt, device=device)
                     for k, (n, dt) in buffer_sizes(plan, c, self.elem).items()}
        self.codes, self.outliers = views["codes"], views["outliers"]
        self.stats, self.hist_seg = views["stats"], views["hist_seg"]
        self.hist_total = views["hist_total"]
        lib = _lib.load()
        wsb = lib.latec_stage_workspace_bytes(plan.handle, c, self.ldtype)
        self.ws = torch.empty(max(int(wsb), 1), dtype=torch.uint8, device=device)
        self.err = torch.zeros(2, dtype=torch.int64, device=device)


def buffer_sizes(plan, c, elem):
    """kind -> (elements, dtype) of the per-call buffers a ``_Buffers`` may
    take as views: codes, outliers, stage statistics, segment and full
    histograms."""
    torch = _torch()
    total = sum(n * c for n in plan.counts)
    segs = sum(-(-(n * c) // rans_model.SEG) for n in plan.counts)
    ns = len(plan)
    return {"codes": (max(total, 1), torch.int16),
            "outliers": (max(total, 1) * elem, torch.uint8),
            "stats": (ns * ctypes.sizeof(_lib.StageStats), torch.uint8),
            "hist_seg": (max(segs, 1) * 2 * rans_model.HWIN, torch.int32),
            "hist_total": (ns * 65536, torch.int32)}


def _qparams(dtype_id, c, radius, order, center, end_mode, round_output):
    return _lib.QuantParams(dtype=_lib.F64 if dtype_id == 2 else _lib.F32, channels=c,
                            radius=int(radius), order=1 if order == "cubic" else 0,
                            center=int(center), end_mode=int(end_mode),
                            round_output=int(bool(round_output)), reserved=0)


# numpy twin of the FitStage descriptor (fit_kernels.cu), field for field
# numpy twin of latec_rans_stage (include/latec_b200.h), field for field
_RANS_DTYPE = np.dtype([(n, np.uint64) for n in ("codes_off", "out_off", "enc", "cdf", "bucket",
                                                 "scratch_off", "blob_off", "rec_off",
                                                 "framed_hi")]
                       + [("n", np.uint32), ("K", np.uint32), ("n_chunks", np.uint32),
                          ("chunk0", np.uint32), ("alphabet", np.uint32), ("kexp", np.int32),
                          ("radius", np.int32), ("mode", np.int32), ("per_point", np.int32),
                          ("blob_words", np.uint32), ("n_out", np.uint32), ("block0", np.uint32)],
                       align=True)
_FIT_DTYPE = np.dtype([("counts_off", np.uint64), ("w_table", np.uint64), ("seg_off", np.uint64),
                       ("n_segs", np.uint32), ("alphabet", np.uint32), ("kexp", np.int32),
                       ("radius", np.int32), ("n_shapes", np.uint32), ("stage", np.uint32),
                       ("shape_ids", np.uint32, (24,))], align=True)


def _stage_flat(plan, t):
    """Flat grid indices of stage t in the reference's order
    (np.flatnonzero of the stage mask)."""
    n = int(plan.counts[t])
    flat = np.empty(n, np.int64)
    if n:
        # host-side plan arithmetic: no device needed (as for the plan itself)
        _lib.check(_lib.load(require_gpu=False).latec_plan_stage_flat(
            plan.handle, t, 0, n, flat.ctypes.data_as(ctypes.c_void_p)), "latec_plan_stage_flat")
    return flat


def _stats_from_device(buf, ns):
    raw = buf.stats.cpu().numpy().tobytes()
    arr = (_lib.StageStats * ns).from_buffer_copy(raw)
    _lib.check_stage_stats(arr)
    return arr


def _check_radius(radius):
    if not 1 <= int(radius) <= 1 << 15:
        raise NotImplementedError(
            f"the CUDA quantizer supports radius in [1, 32768] (16-bit codes); got {radius}")


class _Encoder:
    """One compress call's GPU state: the field, the plan and the buffers."""

    def __init__(self, field, spatial, c, src, levels_, anchor_stride, anchor_block, radius,
                 order, entropy, zstd_level, device, predictor=None):
        self.field, self.spatial, self.c, self.src = field, spatial, c, src
        self.predictor = predictor  # a caller's predictor (None: the fused interpolation)
        self.plan = levels.plan_for(spatial, levels_, anchor_stride, anchor_block)
        self.radius, self.order, self.entropy, self.zstd_level = radius, order, entropy, zstd_level
        self.device = device
        self.buf = _Buffers(self.plan, c, src, device)
        self.mode = _lib.RANS_LANES if entropy == "native" else _lib.RANS_COMPAT
        self.lib = _lib.load()

    def encode(self, ebs, center, end_mode, recon):
        """Run every stage; return (payload uint8 array, per-stage stats dict)."""
        torch = _torch()
        lib, b, plan = self.lib, self.buf, self.plan
        ns = len(plan)
        prm = _qparams(self.src, self.c, self.radius, self.order, center, end_mode,
                       self.src == 0)
        eb_arr = (ctypes.c_double * ns)(*[float(e) for e in ebs])
        stream = _lib.stream_ptr()
        t0 = time.perf_counter()
        if self.predictor is not None:
            recon.zero_()
        if self.predictor is None:
            _lib.check(lib.latec_encode_stages(
                plan.handle, ctypes.byref(prm), eb_arr, self.field.data_ptr(), recon.data_ptr(),
                b.codes.data_ptr(), b.outliers.data_ptr(), b.stats.data_ptr(),
                b.hist_seg.data_ptr(), b.hist_total.data_ptr(), b.ws.data_ptr(), b.ws.numel(),
                stream), "latec_encode_stages")
        else:
            self._caller_stages(ebs, recon, prm, stream)
        st = _stats_from_device(b, ns)
        t1 = time.perf_counter()
        if self.mode == _lib.RANS_LANES:
            fits = self._fit_native(st)
        else:
            fits = self._fit_reference(st)
        t_fit = time.perf_counter()
        # ---- entropy stage on the device
        rs = np.zeros(ns, _RANS_DTYPE)
        keep = []
        kx = np.asarray([f[0] for f in fits], np.int64)
        rs["codes_off"] = rs["out_off"] = np.asarray(b.offsets[:ns], np.uint64)
        rs["n"] = np.asarray(b.items[:ns], np.uint32)
        rs["kexp"], rs["radius"], rs["mode"] = kx, int(self.radius), self.mode
        rs["alphabet"] = (1 << (kx + 1)).astype(np.uint32)
        for t in range(ns):
            kexp, level, shape, owx, bits = fits[t]
            rs["framed_hi"][t] = bitstream.pack_frame(0, kexp, shape, level, owx, False)
            n = int(b.items[t])
            if n:
                cdf, enc, bucket, alphabet = rans_model.device_tables.get(
                    self.mode, kexp, shape, owx, level, self.device)
                keep.append((cdf, enc, bucket))
                rs["cdf"][t], rs["enc"][t], rs["bucket"][t] = (cdf.data_ptr(), enc.data_ptr(),
                                                               bucket.data_ptr())
                if self.mode == _lib.RANS_LANES:
                    rs["K"][t] = rans_model.lanes_K(n, bits)
        stages = rs.ctypes.data
        wsb = lib.latec_rans_encode_workspace_bytes(stages, ns)
        ws = torch.empty(max(int(wsb), 1), dtype=torch.uint8, device=self.device)
        items = np.asarray(b.items[:ns], np.int64)
        cap = int(np.sum(16 + 4 * (1 + 65 * rs["n_chunks"].astype(np.int64) + items + 2)
                         + b.elem * items))
        cap = (cap + 15) // 16 * 16
        payload = torch.empty(cap, dtype=torch.uint8, device=self.device)
        plen = torch.zeros(1, dtype=torch.int64, device=self.device)
        err = torch.zeros(1, dtype=torch.int32, device=self.device)
        _lib.check(lib.latec_rans_encode(
            stages, ns, b.codes.data_ptr(), None, b.stats.data_ptr(), b.outliers.data_ptr(),
            b.elem, payload.data_ptr(), cap, plen.data_ptr(), err.data_ptr(), ws.data_ptr(),
            ws.numel(), stream), "latec_rans_encode")
        # one download: payload length, error word and the stage descriptors
        dsz = ctypes.sizeof(_lib.RansStage) * ns
        tail = torch.cat([plen.view(torch.uint8), err.view(torch.uint8),
                          ws[:dsz]]).cpu().numpy()
        n_bytes = int(tail[:8].view(np.int64)[0])
        e = int(tail[8:12].view(np.int32)[0])
        t_rans = time.perf_counter()
        if e:
            raise RuntimeError(f"entropy coder reported error bits {e:#x}")
        desc = (_lib.RansStage * ns).from_buffer_copy(tail[12:12 + dsz].tobytes())
        rec_bytes = [16 + 4 * int(desc[t].blob_words) + b.elem * int(desc[t].n_out)
                     for t in range(ns)]
        del keep
        stage = dict(
            stage_codes=[int(v) for v in b.items],
            stage_outliers=[int(st[t].n_out) for t in range(ns)],
            stage_payload_bytes=rec_bytes,
            stage_model_bits=[0.0] * ns,
            stage_pred_sae=[float(st[t].stats[0]) for t in range(ns)],
            stage_pred_sse=[float(st[t].stats[1]) for t in range(ns)],
            stage_recon_sae=[float(st[t].stats[2]) for t in range(ns)],
            stage_recon_sse=[float(st[t].stats[3]) for t in range(ns)],
            stage_recon_max=[float(st[t].stats[4]) for t in range(ns)],
            predict_s=t1 - t0, quantize_s=0.0, entropy_s=t_rans - t1,
            fit_s=t_fit - t1, rans_s=t_rans - t_fit,
            outliers=int(sum(int(st[t].n_out) for t in range(ns))),
            stage_fit=fits,
        )
        return payload, n_bytes, stage

    def _caller_stages(self, ebs, recon, prm, stream):
        """The reference's closed loop (``latec/codec.py:384-459``) around a
        caller's predictor: per stage its ``predict(recon, known, pos)`` on
        the host arrays the reference passes (the anchors predicted as 0),
        then the device quantizer writes the stage's codes, outliers,
        statistics and histograms where the fused stage kernels would, and
        its reconstruction returns to ``recon`` and to the host copy."""
        torch = _torch()
        lib, b, plan = self.lib, self.buf, self.plan
        c, spatial = self.c, tuple(self.spatial)
        dt = np.float64 if self.src == 2 else np.float32
        recon_np = np.zeros((c,) + spatial, dt)
        known = np.zeros(spatial, bool)
        flat_field = self.field.reshape(c, -1)
        flat_recon = recon.reshape(c, -1)
        b.stats.zero_()
        b.hist_seg.zero_()
        b.hist_total.zero_()
        ssz = ctypes.sizeof(_lib.StageStats)
        for t in range(len(plan)):
            n = int(plan.counts[t])
            if n == 0:
                continue
            flat = _stage_flat(plan, t)
            pos = np.zeros(int(np.prod(spatial)), bool)
            pos[flat] = True
            pos = pos.reshape(spatial)
            if t == 0:
                pred = np.zeros((c, n), dt)
            else:
                pred = np.asarray(self.predictor.predict(recon_np, known, pos), dt).reshape(c, n)
            idx = torch.from_numpy(flat).to(self.device)
            x = flat_field[:, idx].contiguous()
            p = torch.from_numpy(np.ascontiguousarray(pred)).to(self.device)
            out = torch.empty_like(x)
            items = c * n
            ws = torch.empty(max(int(lib.latec_flat_workspace_bytes(items, b.ldtype)), 1),
                             dtype=torch.uint8, device=self.device)
            off = int(b.offsets[t])
            _lib.check(lib.latec_quantize(
                ctypes.byref(prm), float(ebs[t]), items, x.data_ptr(), p.data_ptr(),
                b.codes.data_ptr() + 2 * off, out.data_ptr(), b.outliers.data_ptr() + b.elem * off,
                b.stats.data_ptr() + t * ssz,
                b.hist_seg.data_ptr() + 4 * 2 * rans_model.HWIN * int(b.seg_off[t]),
                b.hist_total.data_ptr() + 4 * 65536 * t, ws.data_ptr(), ws.numel(), stream),
                "latec_quantize")
            flat_recon[:, idx] = out
            recon_np.reshape(c, -1)[:, flat] = out.cpu().numpy()
            known |= pos

    def _fit_native(self, st):
        """Native-mode stage model fit on the device (fit_kernels.cu)."""
        torch = _torch()
        b, ns = self.buf, len(self.plan)
        idx = [t for t in range(ns) if b.items[t]]
        fits = [(1, 0, 0, 0, 0.0)] * ns
        if not idx:
            return fits
        n = len(idx)
        items = np.asarray([b.items[t] for t in idx], np.int64)
        maxq = np.asarray([int(st[t].maxq) for t in idx], np.int64)
        nout = np.asarray([int(st[t].n_out) for t in idx], np.int64)
        kexps = np.asarray([rans_model.kexp_from_maxq(q) for q in maxq.tolist()], np.int64)
        if np.any(kexps > 15):
            raise ValueError("rANS coder window does not fit the stage frame")
        owxs = rans_model.choose_outlier_weights(nout, items)
        fs = np.zeros(n, _FIT_DTYPE)
        alph = (2 << kexps).astype(np.int64)
        fs["counts_off"] = np.concatenate([[0], np.cumsum(alph)[:-1]])
        fs["seg_off"] = np.asarray([int(b.seg_off[t]) for t in idx], np.uint64)
        fs["n_segs"] = np.asarray([int(b.segs[t]) for t in idx], np.uint32)
        fs["alphabet"], fs["kexp"], fs["radius"] = alph, kexps, int(self.radius)
        fs["stage"] = np.asarray(idx, np.uint32)
        keep, tabs = [], {}
        for key in set(zip(kexps.tolist(), owxs.tolist())):
            w, ids = rans_model.device_weights.get(key[0], key[1], self.device)
            keep.append(w)
            row = np.zeros(24, np.uint32)
            row[:len(ids)] = ids
            tabs[key] = (w.data_ptr(), len(ids), row)
        for j, key in enumerate(zip(kexps.tolist(), owxs.tolist())):
            ptr, nsh, row = tabs[key]
            fs["w_table"][j], fs["n_shapes"][j], fs["shape_ids"][j] = ptr, nsh, row
        meta = list(zip(kexps.tolist(), owxs.tolist()))
        off = int(alph.sum())
        n = len(idx)
        counts = torch.empty(off, dtype=torch.int32, device=self.device)
        costs = torch.empty(n * 24 * 64, dtype=torch.float64, device=self.device)
        out = torch.empty(n * 3, dtype=torch.float64, device=self.device)
        ws = torch.empty(n * ctypes.sizeof(_lib.FitStage) + 256, dtype=torch.uint8, device=self.device)
        _lib.check(self.lib.latec_fit_const(fs.ctypes.data, n, b.hist_seg.data_ptr(), b.hist_total.data_ptr(),
                                            counts.data_ptr(), costs.data_ptr(), out.data_ptr(),
                                            ws.data_ptr(), ws.numel(), _lib.stream_ptr()),
                   "latec_fit_const")
        res = out.cpu().numpy().reshape(n, 3)
        for j, t in enumerate(idx):
            kexp, owx = meta[j]
            fits[t] = (kexp, int(res[j, 1]), int(res[j, 2]), owx, float(res[j, 0]))
        return fits

    def _fit_reference(self, st):
        """The reference's float32 fit on the host (compat streams)."""
        torch = _torch()
        b, ns = self.buf, len(self.plan)
        hist_seg = b.hist_seg.cpu().numpy().view(np.uint32).reshape(-1, 2 * rans_model.HWIN)
        need_total = [t for t in range(ns) if st[t].maxq >= rans_model.HWIN]
        totals = {}
        if need_total:
            rows = b.hist_total.view(ns, 65536)[torch.tensor(need_total, device=self.device)]
            rows = rows.cpu().numpy().view(np.uint32)
            totals = {t: rows[i] for i, t in enumerate(need_total)}
        fits = []
        for t in range(ns):
            n = b.items[t]
            if n == 0:
                fits.append((1, 0, 0, 0, 0.0))
                continue
            kexp = rans_model.kexp_from_maxq(st[t].maxq)
            if kexp > 15:
                raise ValueError("rANS coder window does not fit the stage frame")
            seg = hist_seg[b.seg_off[t]:b.seg_off[t + 1]]
            hist = rans_model.stage_hist_f32(n, kexp, self.radius, seg, totals.get(t))
            level, shape, owx, bits = rans_model.fit_const_level(hist, n, kexp)
            fits.append((kexp, level, shape, owx, bits))
        return fits

    def to_stream(self, payload, n_bytes, header: bytes, stage):
        """Container bytes: native streams are framed on the device and copied
        once through pinned memory; compat streams take the reference's
        literal-zstd decisions and a level-``zstd_level`` zstd frame on the host."""
        torch = _torch()
        t0 = time.perf_counter()
        if self.mode == _lib.RANS_LANES:
            total = len(header) + int(self.lib.latec_raw_frame_bytes(n_bytes))
            hdr = torch.frombuffer(bytearray(header), dtype=torch.uint8).to(self.device)
            out = torch.empty(total, dtype=torch.uint8, device=self.device)
            _lib.check(self.lib.latec_frame_raw(payload.data_ptr(), n_bytes, hdr.data_ptr(),
                                                len(header), out.data_ptr(), total,
                                                _lib.stream_ptr()), "latec_frame_raw")
            if getattr(self, "stream_out", "bytes") == "device":
                stream = out
            elif getattr(self, "stream_out", "bytes") == "numpy":
                host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
                host.copy_(out, non_blocking=True)
                torch.cuda.current_stream().synchronize()
                stream = host.numpy()
            else:
                pin = _lib.pinned(total, "stream_out")
                pin[:total].copy_(out, non_blocking=True)
                torch.cuda.current_stream().synchronize()
                stream = bytes(pin[:total].numpy())
        else:
            host = payload[:n_bytes].cpu().numpy()
            host = self._compat_literals(host, stage["stage_fit"])
            stage["stage_payload_bytes"] = self._record_sizes(host, len(self.plan))
            body = bitstream.zstd().compress(host, self.zstd_level)
            stream = header + body
            n_bytes = len(host)
        stage["entropy_s"] += time.perf_counter() - t0
        stage["download_s"] = time.perf_counter() - t0
        stage["raw_payload_bytes"] = int(n_bytes)
        return stream

    def _record_sizes(self, payload, ns):
        out, off = [], 0
        for _ in range(ns):
            n, word = struct.unpack_from("<IQ", payload, off)
            hlen = word & ((1 << 45) - 1)
            (n_out,) = struct.unpack_from("<I", payload, off + 12 + hlen)
            size = 16 + hlen + self.buf.elem * n_out
            out.append(size)
            off += size
        return out

    def _compat_literals(self, payload, fits):
        """Reference back-end choice for large stages (``latec/bitstream.py:203-219``):
        the narrowed symbols deflated by zstd replace the rANS blob when a
        level-1 scout and then the full-level pass beat the model's bits."""
        b = self.buf
        parts, off = [], 0
        for t in range(len(self.plan)):
            n, word = struct.unpack_from("<IQ", payload, off)
            hlen = word & ((1 << 45) - 1)
            (n_out,) = struct.unpack_from("<I", payload, off + 12 + hlen)
            size = 16 + hlen + b.elem * n_out
            rec = payload[off:off + size]
            kexp, level, shape, owx, bits = fits[t]
            if n >= rans_model.LITERAL_MIN:
                codes = b.codes[b.offsets[t]:b.offsets[t + 1]].cpu().numpy().view(np.uint16)
                syms = rans_model.narrow_literals(codes, self.radius, kexp).tobytes()
                z = bitstream.zstd()
                scout = z.compress(syms, 1)
                if len(scout) * rans_model.LITERAL_SCOUT_SLACK < bits / 8.0:
                    blob = z.compress(syms, self.zstd_level)
                    if len(blob) * 8.0 < bits:
                        head = struct.pack("<IQ", n, bitstream.pack_frame(
                            len(blob), kexp, shape, level, owx, True))
                        tail = rec[12 + hlen:].tobytes()
                        rec = np.frombuffer(head + blob + tail, np.uint8)
            parts.append(np.asarray(rec, np.uint8))
            off += size
        return np.concatenate(parts) if parts else np.zeros(0, np.uint8)


def _finalize(canvas, src_dtype, channels, as_numpy=True):
    """``latec/codec.py:513-524``: (C, *S) -> (*S, C) in the source dtype."""
    torch = _torch()
    out = canvas.movedim(0, -1)
    dt = DTYPE_CODES[src_dtype]
    if np.issubdtype(dt, np.integer):
        info = np.iinfo(dt)
        out = torch.clamp(torch.round(out), info.min, info.max).to(torch.uint8)
    elif dt == np.float64:
        out = out.to(torch.float64)
    else:
        out = out.to(torch.float32)
    if channels == 1:
        out = out[..., 0]
    out = out.contiguous()
    if as_numpy:
        host = torch.empty(out.shape, dtype=out.dtype, pin_memory=True)
        host.copy_(out, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return host.numpy()
    return out


def _is_gpu_interp(predictor):
    return getattr(predictor, "_latec_gpu_interp", False)


def compress(img, eb, predictor, levels=4, anchor_stride=16, anchor_block=1, radius=1 << 15,
             zstd_level=9, eb_ratio=None, tune="fast", tune_size_slack=1.05, verbose=False, *,
             entropy="native", device=None, recon="auto", stream_out="bytes"):
    """Compress an image or an arbitrary-rank scalar field; returns ``(stream, stats)``.

    Mirrors ``latec/codec.py:45-285``. ``img`` may be a NumPy array or a torch
    tensor (host or CUDA). Extra keyword-only options: ``entropy`` ("native" or
    "compat"), ``device`` (CUDA device; default the current one) and ``recon``
    ("auto": ``stats["recon"]`` in the input's kind -- NumPy for NumPy input,
    a device tensor for a CUDA tensor -- or "numpy", "device", "none").
    """
    torch = _torch()
    _lib.load()
    if entropy not in ("native", "compat"):
        raise ValueError("entropy must be 'native' or 'compat'")
    if stream_out not in ("bytes", "device", "numpy"):
        raise ValueError("stream_out must be 'bytes', 'numpy' or 'device'")
    if stream_out != "bytes" and entropy != "native":
        raise ValueError("numpy and device streams use the native entropy mode")
    if not eb > 0:
        raise ValueError(f"error bound must be > 0, got {eb}")
    _check_radius(radius)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    input_is_cuda = _is_tensor(img) and img.is_cuda
    field, spatial, c, src = _prepare(img, dev)
    if len(spatial) > 6:
        raise NotImplementedError("the CUDA codec supports up to 6 spatial axes")
    if field.numel():  # one download for both ends of the range
        mm = torch.aminmax(field)
        vmin, vmax = (float(v) for v in torch.stack([mm.min, mm.max]).double().cpu().tolist())
    else:
        vmin, vmax = 0.0, 0.0
    if not (vmax > vmin):
        if not (np.isnan(vmin) or np.isnan(vmax)):
            vmax = vmin + 1.0
    for name, val in (("levels", levels), ("anchor_stride", anchor_stride),
                      ("anchor_block", anchor_block)):
        got = getattr(predictor, name, val)
        if got != val:
            raise ValueError(f"predictor {name}={got} != compress {name}={val}")
    # any other predictor is the reference's duck-typed plugin: its predict()
    # runs per stage on the host, the quantizer and the coder on the device
    caller = not _is_gpu_interp(predictor)
    if caller and getattr(predictor, "provides_scale", False):
        raise NotImplementedError(
            "per-point scale predictors are coded by GNNCodec (the learned container)")
    from . import levels as _levels

    _levels.check_plan(spatial, levels, anchor_stride, anchor_block)
    order = "linear" if caller else predictor.order
    enc = _Encoder(field, spatial, c, src, levels, anchor_stride, anchor_block, radius, order,
                   entropy, zstd_level, dev, predictor=predictor if caller else None)
    enc.stream_out = stream_out
    flags = getattr(predictor, "stream_flag", 0)
    if entropy == "native":
        flags |= FLAG_LANES

    def ebs_for(ratio):
        return _levels.stage_ebs(spatial, levels, anchor_stride, anchor_block, eb, ratio)

    def make_header(center, ratio, end_mode):
        return Header(channels=c, src_dtype=src, spatial=tuple(spatial), eb=float(eb),
                      levels=levels, anchor_stride=anchor_stride, anchor_block=anchor_block,
                      radius=radius, max_radius=getattr(predictor, "max_radius", 0),
                      agg_level=-1 if getattr(predictor, "agg_level", None) is None
                      else int(predictor.agg_level),
                      vmin=vmin, vmax=vmax,
                      ckpt_hash=getattr(predictor, "checkpoint_hash", b"\0" * 16),
                      flags=flags | (int(end_mode) << END_MODE_SHIFT), interp_center=center,
                      eb_ratio=ratio)

    if tune not in ("fast", "size", "rd"):
        raise ValueError("tune must be 'fast', 'size', or 'rd'")
    tunable = getattr(predictor, "tunable", False)
    nd = len(spatial)
    if not caller and getattr(predictor, "center", None) is None:
        predictor.center = 1 if nd >= 4 else 0
    if not caller and getattr(predictor, "end_mode", None) is None:
        predictor.end_mode = 1
    if eb_ratio is not None:
        ratio_cands = [eb_ratio]
    elif tunable and tune != "fast":
        ratio_cands = [1.0, 0.9, 0.8, 0.7]
    else:
        ratio_cands = [getattr(predictor, "fast_eb_ratio", 1.0)]
    sweep = tunable and tune != "fast" and eb_ratio is None
    base_center = 0 if caller else predictor.center
    center_cands = [base_center] + ([x for x in (0, 1, 2) if x != base_center] if sweep else [])
    base_end = 0 if caller else predictor.end_mode
    candidates = []
    seen = set()

    def run(ratio, center, end_mode):
        rc = torch.empty_like(field)
        payload, n_bytes, st = enc.encode(ebs_for(ratio), center, end_mode, rc)
        stream = enc.to_stream(payload, n_bytes, make_header(center, ratio, end_mode).pack(), st)
        del payload
        st["compressed_bytes"] = len(stream)
        st["recon_sse"] = float(sum(st["stage_recon_sse"]))
        candidates.append((len(stream), st["recon_sse"], ratio, center, end_mode, stream, rc, st))

    def run_once(ratio, center, end_mode):
        if (ratio, center, end_mode) not in seen:
            seen.add((ratio, center, end_mode))
            run(ratio, center, end_mode)

    run_once(ratio_cands[0], base_center, base_end)
    chosen_end = base_end
    if sweep:
        for em in range(END_MODE_MAX + 1):
            run_once(ratio_cands[0], base_center, em)
        chosen_end = min(candidates, key=lambda x: (x[0], x[1]))[4]
    for ratio in ratio_cands:
        for center in center_cands:
            run_once(ratio, center, chosen_end)
    if tune == "rd" and eb_ratio is None and tunable and len(candidates) > 1:
        limit = min(x[0] for x in candidates) * tune_size_slack
        best = min((x for x in candidates if x[0] <= limit),
                   key=lambda x: (x[1], x[0], x[2], x[3], x[4]))
    else:
        best = min(candidates, key=lambda x: (x[0], x[1], x[2], x[3], x[4]))
    _, _, ratio, center, end_mode, stream, canvas, stats = best
    stats["tune_candidates"] = len(candidates)
    stats["search_predict_s"] = sum(x[7]["predict_s"] for x in candidates)
    stats["search_quantize_s"] = sum(x[7]["quantize_s"] for x in candidates)
    stats["search_entropy_s"] = sum(x[7]["entropy_s"] for x in candidates)
    if not caller:
        predictor.center = center
        predictor.end_mode = end_mode
    stats["eb_ratio"] = ratio
    stats["interp_center"] = center
    stats["interp_end_mode"] = end_mode
    stats["tune"] = tune
    stats["tune_size_slack"] = tune_size_slack if (tune == "rd" and eb_ratio is None and tunable) else 1.0
    stats["entropy"] = entropy
    if verbose:
        print(f"tuned: eb_ratio={ratio} center={center} end_mode={end_mode} "
              f"compressed={len(stream)} bytes raw={stats['raw_payload_bytes']} bytes "
              f"sse={stats['recon_sse']:.6g}")
    mode = recon if recon != "auto" else ("device" if input_is_cuda else "numpy")
    if mode == "none":
        stats["recon"] = None
    else:
        stats["recon"] = _finalize(canvas, src, c, as_numpy=(mode == "numpy"))
    nbytes = img.nbytes if not _is_tensor(img) else img.numel() * img.element_size()
    stats["original_bytes"] = int(nbytes)
    stats["ratio"] = nbytes / (stream.numel() if _is_tensor(stream) else len(stream))
    return stream, stats


def _caller_decode(predictor, plan, ebs, prm, codes, offsets, pay_dev, recs, c, spatial,
                   src_dtype, recon, err, dev, sp):
    """The reference's decode loop (``latec/codec.py:462-510``) around a
    caller's predictor: per stage its ``predict(recon, known, pos)`` on the
    host, then the device dequantizer against the decoded codes and the
    stage's outliers (copied out of the payload to an aligned buffer)."""
    torch = _torch()
    lib = _lib.load()
    dt = np.float64 if src_dtype == 2 else np.float32
    esz = 8 if src_dtype == 2 else 4
    recon_np = np.zeros((c,) + tuple(spatial), dt)
    known = np.zeros(tuple(spatial), bool)
    flat_recon = recon.reshape(c, -1)
    for t in range(len(plan)):
        n = int(plan.counts[t])
        if n == 0:
            continue
        flat = _stage_flat(plan, t)
        pos = np.zeros(int(np.prod(spatial)), bool)
        pos[flat] = True
        pos = pos.reshape(tuple(spatial))
        if t == 0:
            pred = np.zeros((c, n), dt)
        else:
            pred = np.asarray(predictor.predict(recon_np, known, pos), dt).reshape(c, n)
        p = torch.from_numpy(np.ascontiguousarray(pred)).to(dev)
        n_o = int(recs[t].n_out)
        a = int(recs[t].out_at)
        outl = (pay_dev[a:a + esz * n_o].clone() if n_o
                else torch.zeros(esz, dtype=torch.uint8, device=dev))
        items = c * n
        out = torch.empty((c, n), dtype=recon.dtype, device=dev)
        ws = torch.empty(max(int(lib.latec_dequantize_workspace_bytes(items)), 1),
                         dtype=torch.uint8, device=dev)
        _lib.check(lib.latec_dequantize(ctypes.byref(prm), float(ebs[t]), items, p.data_ptr(),
                                        codes.data_ptr() + 2 * int(offsets[t]), outl.data_ptr(),
                                        n_o, out.data_ptr(), err.data_ptr(), ws.data_ptr(),
                                        ws.numel(), sp), "latec_dequantize")
        flat_recon[:, torch.from_numpy(flat).to(dev)] = out
        recon_np.reshape(c, -1)[:, flat] = out.cpu().numpy()
        known |= pos


def _upload_stream(body, dev):
    """Host bytes -> device: one DMA from page-locked memory, else through a
    pinned staging buffer."""
    torch = _torch()
    n = len(body)
    if isinstance(body, np.ndarray) and body.flags.writeable and n:
        t = torch.from_numpy(body)
        if t.is_pinned():
            d = torch.empty(n + 4, dtype=torch.uint8, device=dev)
            d[:n].copy_(t, non_blocking=True)
            d[n:].zero_()
            return d
    pin = _lib.pinned(n + 4, "stream_in")
    pin.numpy()[:n] = body
    d = torch.empty(n + 4, dtype=torch.uint8, device=dev)
    d[:n].copy_(pin[:n], non_blocking=True)
    d[n:].zero_()
    return d


def _raw_frame_size(head13: bytes, n_body: int):
    """Payload size when the body is a raw-block frame of the native layout."""
    if len(head13) < 13 or head13[:5] != struct.pack("<IB", 0xFD2FB528, 0xE0):
        return None
    (n,) = struct.unpack_from("<Q", head13, 5)
    nblk = max(1, -(-n // (1 << 17)))
    return int(n) if n_body == 13 + 3 * nblk + n else None


_STATUS = {1: "truncated stage record", 2: "truncated stage record", 3: "truncated stage record",
           4: "rANS payload is not aligned to 32-bit words", 5: "lane coder blob has K = 0",
           6: "truncated lane-coder chunk table", 7: "trailing data after the last stage record"}


def decompress(stream, predictor_factory=None, *, device=None, out="numpy"):
    """Decompress a LATEC stream (``latec/codec.py:288-322``).

    ``stream`` is ``bytes`` (or any buffer) or a CUDA ``uint8`` tensor; the
    stage records are parsed, entropy-decoded and dequantized on the device.
    ``out="device"`` returns a CUDA tensor instead of a NumPy array."""
    torch = _torch()
    lib = _lib.load()
    from . import levels as _levels
    from .predictor import InterpPredictor

    is_dev = _is_tensor(stream) and stream.is_cuda
    if is_dev:
        if stream.dtype != torch.uint8 or stream.dim() != 1:
            raise ValueError("a device stream must be a 1-D uint8 tensor")
        n_total = stream.numel()
        prefix = stream[:min(n_total, 4096)].cpu().numpy().tobytes()
        dev = stream.device
    else:
        mv = memoryview(stream).cast("B")
        n_total = len(mv)
        np_stream = stream if isinstance(stream, np.ndarray) else None
        prefix = mv[:min(n_total, 4096)].tobytes()
        dev = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
    header = Header.unpack(prefix)
    if header.flags & FLAG_RANS:
        raise NotImplementedError("per-point scale streams are decoded by GNNCodec.uncompress")
    if predictor_factory is None:
        if header.flags & FLAG_INTERP:
            predictor_factory = lambda hdr: InterpPredictor(  # noqa: E731
                "cubic" if hdr.flags & FLAG_CUBIC else "linear", hdr.levels, hdr.anchor_stride,
                hdr.anchor_block)
        else:
            raise ValueError("stream needs a predictor_factory")
    predictor = predictor_factory(header)
    if hasattr(predictor, "center"):
        predictor.center = header.interp_center
    if hasattr(predictor, "end_mode"):
        predictor.end_mode = (header.flags >> END_MODE_SHIFT) & END_MODE_MAX
    caller = not _is_gpu_interp(predictor)  # a caller's predictor: predict() per stage
    if caller and getattr(predictor, "provides_scale", False):
        raise NotImplementedError("per-point scale predictors are decoded by GNNCodec")
    if header.src_dtype not in DTYPE_CODES:
        raise KeyError(header.src_dtype)
    _check_radius(header.radius)
    spatial, c = tuple(header.spatial), int(header.channels)
    if c < 1:
        raise ValueError("stream has no channels")
    plan = _levels.plan_for(spatial, header.levels, header.anchor_stride, header.anchor_block)
    ns = len(plan)
    ebs = _levels.stage_ebs(spatial, header.levels, header.anchor_stride, header.anchor_block,
                            header.eb, header.eb_ratio)
    elem = 8 if header.src_dtype == 2 else 4
    mode = _lib.RANS_LANES if header.flags & FLAG_LANES else _lib.RANS_COMPAT
    sp = _lib.stream_ptr()
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    # ---- payload on the device
    n_body = n_total - header.size
    n_raw = _raw_frame_size(prefix[header.size:header.size + 13], n_body)
    if n_raw is not None:
        if is_dev:
            frame_dev = stream[header.size:]
        else:
            body_np = (np_stream.reshape(-1)[header.size:] if np_stream is not None
                       else np.frombuffer(mv[header.size:], np.uint8))
            frame_dev = _upload_stream(body_np, dev)
        n_pay = n_raw
        pay_dev = torch.zeros(n_pay + 8 + (-n_pay) % 4, dtype=torch.uint8, device=dev)
        _lib.check(lib.latec_unframe_raw(frame_dev.data_ptr(), n_pay, pay_dev.data_ptr(),
                                         err.data_ptr(), sp), "latec_unframe_raw")
        del frame_dev
    else:
        body = (stream[header.size:].cpu().numpy() if is_dev
                else np.frombuffer(mv[header.size:], np.uint8))
        payload = bitstream.zstd().decompress_into(body)
        n_pay = len(payload)
        pay_dev = _upload_stream(payload, dev)
    # ---- stage records, parsed on the device
    rec_dev = torch.empty(ns * ctypes.sizeof(_lib.Record), dtype=torch.uint8, device=dev)
    tc_dev = torch.zeros(1, dtype=torch.int64, device=dev)
    _lib.check(lib.latec_parse_records(pay_dev.data_ptr(), n_pay, ns, elem,
                                       int(mode == _lib.RANS_LANES), rec_dev.data_ptr(),
                                       tc_dev.data_ptr(), sp), "latec_parse_records")
    # one download: the records, the chunk total and the error word
    rsz = ns * ctypes.sizeof(_lib.Record)
    got = torch.cat([rec_dev, tc_dev.view(torch.uint8), err.view(torch.uint8)]).cpu().numpy()
    recs = (_lib.Record * ns).from_buffer_copy(got[:rsz].tobytes())
    total_chunks = int(got[rsz:rsz + 8].view(np.int64)[0])
    if int(got[rsz + 8:rsz + 12].view(np.int32)[0]) & 64:  # err is int32
        raise ValueError("zstd frame is corrupt")
    items = [n * c for n in plan.counts]
    offsets = np.concatenate([[0], np.cumsum(items)]).astype(np.int64)
    frames = []
    for t in range(ns):
        if recs[t].status:
            raise ValueError(_STATUS.get(recs[t].status, "malformed stage record"))
        f = bitstream.unpack_frame(int(recs[t].frame))
        if recs[t].n != items[t]:
            raise ValueError("stage code count mismatch")
        if not f["kexp"]:
            raise ValueError("rANS stage record has no coder window")
        if recs[t].n == 0 and f["hlen"]:
            raise ValueError("non-empty rANS blob for an empty stage")
        frames.append(f)
    aligned = all(recs[t].blob % 4 == 0 for t in range(ns) if not frames[t]["literal"])
    blob_word = [recs[t].blob // 4 for t in range(ns)]
    words_dev = pay_dev
    if not aligned:  # literal stages broke the word alignment: gather the rANS blobs
        pieces, at = [], 0
        for t in range(ns):
            nw = 0 if frames[t]["literal"] else -(-frames[t]["hlen"] // 4)
            pieces.append(pay_dev[recs[t].blob:recs[t].blob + 4 * nw])
            blob_word[t] = at
            at += nw
        words_dev = torch.cat(pieces + [torch.zeros(8, dtype=torch.uint8, device=dev)])
    ranges = None
    if mode == _lib.RANS_LANES and total_chunks:
        ranges = torch.empty(2 * total_chunks, dtype=torch.int64, device=dev)
        _lib.check(lib.latec_chunk_ranges(words_dev.data_ptr(), rec_dev.data_ptr(), ns,
                                          ranges.data_ptr(), err.data_ptr(), sp),
                   "latec_chunk_ranges")
    stages = (_lib.RansStage * ns)()
    keep, literal_codes = [], {}
    for t in range(ns):
        r, f, d = recs[t], frames[t], stages[t]
        d.codes_off = int(offsets[t])
        d.n = r.n
        d.kexp, d.radius, d.mode = f["kexp"], int(header.radius), mode
        d.alphabet = 1 << (f["kexp"] + 1)
        d.chunk0, d.n_chunks, d.K = r.chunk0, r.n_chunks, r.K
        if r.n == 0:
            continue
        if f["literal"]:
            blob = pay_dev[r.blob:r.blob + f["hlen"]].cpu().numpy()
            syms = np.frombuffer(bitstream.zstd().decompress_into(blob).tobytes(),
                                 rans_model.literal_dtype(f["kexp"]), count=r.n)
            literal_codes[t] = rans_model.widen(syms, header.radius, f["kexp"]).astype(np.uint16)
            d.n = 0
            continue
        if f["hlen"] % 4:
            raise ValueError("rANS payload is not aligned to 32-bit words")
        cdf, enc, bucket, _ = rans_model.device_tables.get(mode, f["kexp"], f["shape"], f["owx"],
                                                           f["level"], dev)
        keep.append((cdf, enc, bucket))
        d.cdf, d.enc, d.bucket = cdf.data_ptr(), enc.data_ptr(), bucket.data_ptr()
        d.blob_off = blob_word[t]
        d.blob_words = f["hlen"] // 4
    codes = torch.empty(max(int(offsets[-1]), 1), dtype=torch.int16, device=dev)
    ws = torch.empty(int(lib.latec_rans_decode_workspace_bytes(ns)), dtype=torch.uint8, device=dev)
    _lib.check(lib.latec_rans_decode(stages, ns, total_chunks, words_dev.data_ptr(),
                                     ranges.data_ptr() if ranges is not None else None, None,
                                     codes.data_ptr(), err.data_ptr(), ws.data_ptr(), ws.numel(),
                                     sp), "latec_rans_decode")
    for t, lc in literal_codes.items():
        codes[int(offsets[t]):int(offsets[t + 1])].copy_(torch.from_numpy(lc.view(np.int16)).to(dev))
    ldt = _lib.F64 if header.src_dtype == 2 else _lib.F32
    if caller:
        prm = _qparams(header.src_dtype, c, header.radius, "linear", 0, 0, header.src_dtype == 0)
    else:
        prm = _qparams(header.src_dtype, c, header.radius, predictor.order, predictor.center,
                       predictor.end_mode, header.src_dtype == 0)
    ft = torch.float64 if header.src_dtype == 2 else torch.float32
    recon = torch.empty((c,) + spatial, dtype=ft, device=dev)  # every point is decoded
    eb_arr = (ctypes.c_double * ns)(*[float(e) for e in ebs])
    out_off = (ctypes.c_uint64 * ns)(*[recs[t].out_at for t in range(ns)])
    n_out = (ctypes.c_uint32 * ns)(*[recs[t].n_out for t in range(ns)])
    ws2 = torch.empty(max(int(lib.latec_stage_workspace_bytes(plan.handle, c, ldt)), 1),
                      dtype=torch.uint8, device=dev)
    if caller:
        _caller_decode(predictor, plan, ebs, prm, codes, offsets, pay_dev, recs, c, spatial,
                       header.src_dtype, recon, err, dev, sp)
    else:
        _lib.check(lib.latec_decode_stages(plan.handle, ctypes.byref(prm), eb_arr,
                                           codes.data_ptr(), pay_dev.data_ptr(), out_off, n_out,
                                           recon.data_ptr(), err.data_ptr(), ws2.data_ptr(),
                                           ws2.numel(), sp), "latec_decode_stages")
    e = int(err.item())
    del keep
    if e & 1:
        raise ValueError("outlier count mismatch")
    if e & (4 | 8 | 128):
        raise ValueError("trailing data in rANS payload")
    if e & 16:
        raise ValueError("malformed rANS payload")
    if e:
        raise ValueError(f"malformed stream (error bits {e:#x})")
    return _finalize(recon, header.src_dtype, c, as_numpy=(out == "numpy"))
