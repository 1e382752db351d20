"""Many tensors per call: ``compress_many`` / ``decompress_many``.

The reference codes one tensor per call (a serial loop is its batch form).
Here a list of tensors of any shapes and dtypes goes through each phase of
the plain codec together:

* compress: the stage kernels of every tensor are launched back to back
  (no host round trip between tensors); one download brings every stage's
  statistics; one launch fits the stage-constant rANS models of every stage
  of every tensor; one launch per outlier width entropy-codes all of them
  with the 32-lane coder and assembles their records; one frame launch per
  stream and, for host streams, one download. Each stream is byte-identical
  to ``compress(x, eb, predictor, ..., tune="fast")``'s.
* decompress: the payloads are unframed and their records parsed per
  stream, one download brings every record, one launch rANS-decodes every
  stage of every stream, then each field is rebuilt by its stage kernels.

The batching matters most for the entropy stage: a smooth field codes at a
fraction of a bit per value, so its stages split into few lane chunks whose
serial chains leave most SMs idle; the chunks of many tensors in one launch
fill the GPU. Codes, outliers, statistics and histograms of the tensors of a
call live in shared device buffers (about 2 x the input bytes + 5.5 MB per
tensor, beside the inputs and their reconstructions), so callers size their
batches to the memory they have. Only the native entropy mode is batched: a
compat stream given to ``decompress_many`` is decoded on its own.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib, bitstream, levels as _levels, rans_model
from .bitstream import END_MODE_SHIFT, FLAG_CUBIC, FLAG_INTERP, FLAG_LANES, FLAG_RANS, Header
from .codec import (_FIT_DTYPE, _RANS_DTYPE, _STATUS, END_MODE_MAX, _Buffers, _check_radius,
                    _finalize, _is_gpu_interp, _prepare, _qparams, _raw_frame_size, _torch,
                    buffer_sizes, decompress)

__all__ = ["compress_many", "decompress_many", "autotune_many", "cta_caps"]

_ALIGN = 256  # bytes: every tensor's slice of a shared buffer starts on this boundary
_FIT_ROWS = 32768  # stages per model-fit launch

# Encode CTAs per stage for the tensors of a class (rank, value bytes, size
# class), chosen by autotune_many from timed trials; a class without an entry
# takes the single-tensor grid (0). Any cap gives the same streams.
_SIZE_BOUNDS = (1 << 16, 1 << 19, 1 << 22)  # points: < 64 Ki, < 512 Ki, < 4 Mi, larger
_CTA_CANDIDATES = (148, 296, 592, 1184)
_cta_caps: dict = {}


def size_class(points):
    """The size class of a tensor of ``points`` values (0 .. 3)."""
    return sum(int(points) >= b for b in _SIZE_BOUNDS)


def cta_caps():
    """The autotuned table: {(rank, value bytes, size class): encode CTAs}."""
    return dict(_cta_caps)


def cta_cap(ndim, elem, points, caps=None):
    table = _cta_caps if caps is None else caps
    return int(table.get((int(ndim), int(elem), size_class(points)), 0))


class _View:
    """A tensor's slice of a shared buffer, as the kernels see it: an address
    and a length (the buffer itself is kept alive by the caller)."""

    __slots__ = ("ptr", "n")

    def __init__(self, ptr, n):
        self.ptr, self.n = ptr, n

    def data_ptr(self):
        return self.ptr

    def numel(self):
        return self.n


def _arenas(sizes, device):
    """Shared buffers for per-tensor size dicts (kind -> (elements, dtype)):
    returns (per-tensor views, kind -> (buffer, per-tensor element offsets)).
    Statistics and full-histogram rows are packed without gaps, so a stage's
    global index is its tensor's first stage plus its own index; segment
    histograms start on a whole segment row; everything else on an
    ``_ALIGN``-byte boundary."""
    torch = _torch()
    views = [dict() for _ in sizes]
    bufs = {}
    for kind in sizes[0]:
        dt = sizes[0][kind][1]
        esz = torch.empty(0, dtype=dt).element_size()
        unit = {"stats": 1, "hist_total": 1,
                "hist_seg": 2 * rans_model.HWIN}.get(kind, _ALIGN // esz)
        ns = [sz[kind][0] for sz in sizes]
        padded = [-(-n // unit) * unit for n in ns]
        offs = np.concatenate([[0], np.cumsum(padded)[:-1]]).astype(np.int64).tolist()
        buf = torch.empty(max(sum(padded), 1), dtype=dt, device=device)
        base = buf.data_ptr()
        for j, n in enumerate(ns):
            views[j][kind] = _View(base + offs[j] * esz, n)
        bufs[kind] = (buf, offs)
    return views, bufs


class _Job:
    """One tensor of a ``compress_many`` call and the settings ``compress``
    would resolve for it with ``tune="fast"``."""

    def __init__(self, index, img, eb, predictor, lv, stride, block, radius, eb_ratio, device):
        self.index = index
        self.field, self.spatial, self.c, self.src = _prepare(img, device)
        if len(self.spatial) > 6:
            raise NotImplementedError("the CUDA codec supports up to 6 spatial axes")
        _levels.check_plan(self.spatial, lv, stride, block)
        self.lv, self.stride, self.block, self.radius = lv, stride, block, int(radius)
        self.plan = _levels.plan_for(self.spatial, lv, stride, block)
        self.elem = 8 if self.src == 2 else 4
        self.eb = float(eb)
        if not self.eb > 0:
            raise ValueError(f"error bound must be > 0, got {eb}")
        nd = len(self.spatial)
        pc, pe = getattr(predictor, "center", None), getattr(predictor, "end_mode", None)
        self.center = pc if pc is not None else (1 if nd >= 4 else 0)
        self.end_mode = pe if pe is not None else 1
        self.ratio = (eb_ratio if eb_ratio is not None
                      else getattr(predictor, "fast_eb_ratio", 1.0))
        self.ebs = _levels.stage_ebs(self.spatial, lv, stride, block, self.eb, self.ratio)

    def header(self, predictor):
        """The LATEC001 header ``compress`` writes for this tensor."""
        flags = getattr(predictor, "stream_flag", 0) | FLAG_LANES
        return Header(channels=self.c, src_dtype=self.src, spatial=tuple(self.spatial),
                      eb=self.eb, levels=self.lv, anchor_stride=self.stride,
                      anchor_block=self.block, radius=self.radius,
                      max_radius=getattr(predictor, "max_radius", 0),
                      agg_level=-1 if getattr(predictor, "agg_level", None) is None
                      else int(predictor.agg_level),
                      vmin=self.vmin, vmax=self.vmax,
                      ckpt_hash=getattr(predictor, "checkpoint_hash", b"\0" * 16),
                      flags=flags | (int(self.end_mode) << END_MODE_SHIFT),
                      interp_center=self.center, eb_ratio=self.ratio).pack()


def compress_many(tensors, eb, predictor, levels=4, anchor_stride=16, anchor_block=1,
                  radius=1 << 15, eb_ratio=None, *, device=None, stream_out="bytes"):
    """Compress a list of fields; returns their streams in order. ``eb`` is
    one bound for all or a sequence of one per tensor. Each stream equals
    ``compress(x, eb, predictor, levels, anchor_stride, anchor_block, radius,
    eb_ratio=eb_ratio, tune="fast")[0]`` for a predictor in the same state;
    ``predictor`` is not modified. ``stream_out``: "bytes" or "device" (one
    uint8 view of a shared device buffer per stream)."""
    torch = _torch()
    lib = _lib.load()
    if stream_out not in ("bytes", "device"):
        raise ValueError("stream_out must be 'bytes' or 'device'")
    _check_radius(radius)
    if not _is_gpu_interp(predictor):
        raise NotImplementedError("compress_many runs InterpPredictor stages on the device")
    for name, val in (("levels", levels), ("anchor_stride", anchor_stride),
                      ("anchor_block", anchor_block)):
        got = getattr(predictor, name, val)
        if got != val:
            raise ValueError(f"predictor {name}={got} != compress {name}={val}")
    tensors = list(tensors)
    if not tensors:
        return []
    ebs = [eb] * len(tensors) if np.isscalar(eb) else list(eb)
    if len(ebs) != len(tensors):
        raise ValueError("one error bound per tensor")
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    jobs = [_Job(j, x, e, predictor, levels, anchor_stride, anchor_block, radius, eb_ratio, dev)
            for j, (x, e) in enumerate(zip(tensors, ebs))]
    # the data ranges of the headers: one download for all
    mm = []
    for jb in jobs:
        if jb.field.numel():
            m = torch.aminmax(jb.field)
            mm.append(torch.stack([m.min, m.max]).double())
        else:
            mm.append(torch.zeros(2, dtype=torch.float64, device=dev))
    for jb, (lo, hi) in zip(jobs, torch.stack(mm).cpu().tolist()):
        if not (hi > lo) and not (np.isnan(lo) or np.isnan(hi)):
            hi = lo + 1.0
        jb.vmin, jb.vmax = lo, hi
    out = [None] * len(jobs)
    for elem in (4, 8):  # one entropy launch per outlier width
        group = [jb for jb in jobs if jb.elem == elem]
        if group:
            for jb, s in zip(group, _compress_group(group, predictor, dev, lib)):
                out[jb.index] = s
    if stream_out == "bytes":
        return _download(out)
    return out



def autotune_many(tensors, eb, predictor, levels=4, anchor_stride=16, anchor_block=1,
                  radius=1 << 15, eb_ratio=None, *, device=None, per_class=64, repeats=3,
                  candidates=_CTA_CANDIDATES):
    """Choose the encode CTAs per stage of each tensor class (rank, value
    bytes, size class) present in ``tensors`` for ``compress_many``: the
    stage pass of up to ``per_class`` tensors of the class is timed (CUDA
    events, best of ``repeats``) at each candidate cap, and the fastest is
    kept in the table ``compress_many`` reads. Returns {class: (cap, ms)}."""
    torch = _torch()
    lib = _lib.load()
    if not _is_gpu_interp(predictor):
        raise NotImplementedError("autotune_many times InterpPredictor stages on the device")
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    groups = {}
    for x in tensors:
        jb = _Job(0, x, eb, predictor, levels, anchor_stride, anchor_block, radius, eb_ratio, dev)
        key = (len(jb.spatial), jb.elem, size_class(jb.field.numel()))
        if len(groups.setdefault(key, [])) < per_class:
            groups[key].append(jb)
    out = {}
    for key, jobs in sorted(groups.items()):
        # the shared buffers stay referenced (bufs) while the trials run: the
        # views hold raw addresses only
        views, bufs = _arenas([buffer_sizes(jb.plan, jb.c, jb.elem) for jb in jobs], dev)
        esz = jobs[0].field.element_size()
        rsz = [-(-jb.field.numel() * esz // _ALIGN) * _ALIGN for jb in jobs]
        recon = torch.empty(max(sum(rsz), 1), dtype=torch.uint8, device=dev)
        roff = np.concatenate([[0], np.cumsum(rsz)[:-1]]).astype(np.int64).tolist()
        for jb, v, ro in zip(jobs, views, roff):
            jb.buf = _Buffers(jb.plan, jb.c, jb.src, dev, views=v)
            jb.recon = _View(recon.data_ptr() + ro, jb.field.numel())
        best = None
        for cap in candidates:
            caps = {key: int(cap)}
            _stage_pass(jobs, predictor, dev, lib, caps)  # warm-up
            ms = []
            for _ in range(repeats):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                _stage_pass(jobs, predictor, dev, lib, caps)
                b.record()
                b.synchronize()
                ms.append(a.elapsed_time(b))
            t = min(ms)
            if best is None or t < best[1]:
                best = (int(cap), t)
        torch.cuda.synchronize()
        for jb in jobs:
            del jb.buf, jb.recon
        del bufs, recon
        _cta_caps[key] = best[0]
        out[key] = best
    return out

def _download(views):
    """Device streams -> bytes, through one pinned buffer and one wait."""
    torch = _torch()
    lens = [int(v.numel()) for v in views]
    off = np.cumsum([0] + lens)
    pin = torch.empty(max(int(off[-1]), 1), dtype=torch.uint8, pin_memory=True)
    for v, a in zip(views, off[:-1].tolist()):
        pin[a:a + v.numel()].copy_(v, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    host = pin.numpy()
    return [host[a:b].tobytes() for a, b in zip(off[:-1].tolist(), off[1:].tolist())]


def _compress_group(jobs, predictor, dev, lib):
    torch = _torch()
    sp = _lib.stream_ptr()
    views, bufs = _arenas([buffer_sizes(jb.plan, jb.c, jb.elem) for jb in jobs], dev)
    ssz = ctypes.sizeof(_lib.StageStats)
    # the reconstructions the stage kernels work in: one buffer (every
    # point is written)
    esz = jobs[0].field.element_size()
    rsz = [-(-jb.field.numel() * esz // _ALIGN) * _ALIGN for jb in jobs]
    recon = torch.empty(max(sum(rsz), 1), dtype=torch.uint8, device=dev)
    roff = np.concatenate([[0], np.cumsum(rsz)[:-1]]).astype(np.int64).tolist()
    for jb, v, ro in zip(jobs, views, roff):
        jb.buf = _Buffers(jb.plan, jb.c, jb.src, dev, views=v)
        jb.recon = _View(recon.data_ptr() + ro, jb.field.numel())
    _stage_pass(jobs, predictor, dev, lib)
    raw = bufs["stats"][0].cpu().numpy().tobytes()  # one download: every stage's statistics
    stage0 = np.cumsum([0] + [len(jb.plan) for jb in jobs]).tolist()
    for j, jb in enumerate(jobs):
        ns = len(jb.plan)
        jb.st = (_lib.StageStats * ns).from_buffer_copy(raw[stage0[j] * ssz:(stage0[j] + ns) * ssz])
        _lib.check_stage_stats(jb.st)
    _fit_all(jobs, bufs, stage0, dev, lib)
    payload, starts, lens = _entropy_all(jobs, bufs, dev, lib)
    # ---- frames: the headers uploaded together, one frame launch per stream
    heads = [jb.header(predictor) for jb in jobs]
    hoff = np.cumsum([0] + [len(h) for h in heads]).tolist()
    hdev = torch.frombuffer(bytearray(b"".join(heads)), dtype=torch.uint8).to(dev)
    totals = [len(h) + int(lib.latec_raw_frame_bytes(n)) for h, n in zip(heads, lens)]
    soff = np.cumsum([0] + totals).tolist()
    streams = torch.empty(max(soff[-1], 1), dtype=torch.uint8, device=dev)
    for j in range(len(jobs)):
        _lib.check(lib.latec_frame_raw(payload.data_ptr() + starts[j], lens[j],
                                       hdev.data_ptr() + hoff[j], len(heads[j]),
                                       streams.data_ptr() + soff[j], totals[j], sp),
                   "latec_frame_raw")
    for jb in jobs:
        del jb.buf, jb.recon
    return [streams[soff[j]:soff[j + 1]] for j in range(len(jobs))]



def _stage_pass(jobs, predictor, dev, lib, caps=None):
    """Every stage of every tensor (buffers set up in ``jb.buf``, ``jb.recon``):
    stage index by stage index, one launch per kernel class over all tensors
    (latec_encode_stages_many). ``caps``: encode CTAs per stage by tensor
    class, default the autotuned table."""
    torch = _torch()
    ej = (_lib.EncodeJob * len(jobs))()
    keep = []
    for k, jb in enumerate(jobs):
        b = jb.buf
        e = ej[k]
        e.plan = jb.plan.handle
        e.prm = _qparams(jb.src, jb.c, jb.radius, predictor.order, jb.center, jb.end_mode,
                         jb.src == 0)
        eb_arr = (ctypes.c_double * len(jb.plan))(*[float(x) for x in jb.ebs])
        keep.append(eb_arr)
        e.stage_eb = ctypes.addressof(eb_arr)
        e.x, e.recon = jb.field.data_ptr(), jb.recon.data_ptr()
        e.codes, e.outliers = b.codes.data_ptr(), b.outliers.data_ptr()
        e.stats, e.hist_seg, e.hist_total = (b.stats.data_ptr(), b.hist_seg.data_ptr(),
                                             b.hist_total.data_ptr())
        e.workspace, e.workspace_bytes = b.ws.data_ptr(), b.ws.numel()
        e.max_ctas = cta_cap(len(jb.spatial), jb.elem, jb.field.numel(), caps)
    tb = int(lib.latec_encode_many_table_bytes(ej, len(jobs)))
    if not tb:
        raise ValueError("latec_encode_many_table_bytes: invalid job")
    table = torch.empty(tb, dtype=torch.uint8, device=dev)
    _lib.check(lib.latec_encode_stages_many(ej, len(jobs), table.data_ptr(), tb,
                                            _lib.stream_ptr()), "latec_encode_stages_many")
    del keep

def _fit_all(jobs, bufs, stage0, dev, lib):
    """The native stage-model fit (the rule of ``codec._Encoder._fit_native``)
    of every non-empty stage of every tensor in one launch; sets ``jb.fits``."""
    torch = _torch()
    seg_buf, seg_offs = bufs["hist_seg"]
    tot_buf = bufs["hist_total"][0]
    rows = []  # (job, stage, global segment row, segments, kexp, owx, global stage)
    for j, jb in enumerate(jobs):
        b, ns = jb.buf, len(jb.plan)
        jb.fits = [(1, 0, 0, 0, 0.0)] * ns
        idx = [t for t in range(ns) if b.items[t]]
        if not idx:
            continue
        items = np.asarray([b.items[t] for t in idx], np.int64)
        maxq = [int(jb.st[t].maxq) for t in idx]
        nout = np.asarray([int(jb.st[t].n_out) for t in idx], np.int64)
        kexps = [rans_model.kexp_from_maxq(q) for q in maxq]
        if max(kexps) > 15:
            raise ValueError("rANS coder window does not fit the stage frame")
        owxs = rans_model.choose_outlier_weights(nout, items).tolist()
        row0 = seg_offs[j] // (2 * rans_model.HWIN)
        for t, k, o in zip(idx, kexps, owxs):
            rows.append((jb, t, row0 + int(b.seg_off[t]), int(b.segs[t]), int(k), int(o),
                         stage0[j] + t))
    if not rows:
        return
    n = len(rows)
    fs = np.zeros(n, _FIT_DTYPE)
    kx = np.asarray([r[4] for r in rows], np.int64)
    alph = (2 << kx).astype(np.int64)
    fs["counts_off"] = np.concatenate([[0], np.cumsum(alph)[:-1]])
    fs["seg_off"] = np.asarray([r[2] for r in rows], np.uint64)
    fs["n_segs"] = np.asarray([r[3] for r in rows], np.uint32)
    fs["alphabet"], fs["kexp"] = alph, kx
    fs["radius"] = np.asarray([r[0].radius for r in rows], np.int32)
    fs["stage"] = np.asarray([r[6] for r in rows], np.uint32)
    keep, tabs = [], {}
    for key in {(r[4], r[5]) for r in rows}:
        w, ids = rans_model.device_weights.get(key[0], key[1], dev)
        keep.append(w)
        ids_row = np.zeros(24, np.uint32)
        ids_row[:len(ids)] = ids
        tabs[key] = (w.data_ptr(), len(ids), ids_row)
    for i, r in enumerate(rows):
        ptr, nsh, ids_row = tabs[(r[4], r[5])]
        fs["w_table"][i], fs["n_shapes"][i], fs["shape_ids"][i] = ptr, nsh, ids_row
    res = torch.empty(n * 3, dtype=torch.float64, device=dev)
    for a in range(0, n, _FIT_ROWS):  # the fit grid holds at most 65,535 stages per launch
        m = min(_FIT_ROWS, n - a)
        part = np.ascontiguousarray(fs[a:a + m])
        part["counts_off"] -= part["counts_off"][0]
        counts = torch.empty(int(alph[a:a + m].sum()), dtype=torch.int32, device=dev)
        costs = torch.empty(m * 24 * 64, dtype=torch.float64, device=dev)
        ws = torch.empty(m * ctypes.sizeof(_lib.FitStage) + 256, dtype=torch.uint8, device=dev)
        _lib.check(lib.latec_fit_const(part.ctypes.data, m, seg_buf.data_ptr(),
                                       tot_buf.data_ptr(), counts.data_ptr(), costs.data_ptr(),
                                       res.data_ptr() + 24 * a, ws.data_ptr(), ws.numel(),
                                       _lib.stream_ptr()), "latec_fit_const")
    got = res.cpu().numpy().reshape(n, 3)  # one download: every stage's model
    for i, r in enumerate(rows):
        r[0].fits[r[1]] = (r[4], int(got[i, 1]), int(got[i, 2]), r[5], float(got[i, 0]))
    del keep


def _entropy_all(jobs, bufs, dev, lib):
    """Every stage of every tensor through the lane coder and the record
    assembly in one call; returns (payload, each tensor's first byte, each
    tensor's payload bytes)."""
    torch = _torch()
    codes_buf, codes_offs = bufs["codes"]
    out_buf, out_offs = bufs["outliers"]
    stats_buf = bufs["stats"][0]
    elem = jobs[0].elem
    n_all = sum(len(jb.plan) for jb in jobs)
    rs = np.zeros(n_all, _RANS_DTYPE)
    keep, first, cap = [], [], 0
    at = 0
    for j, jb in enumerate(jobs):
        b, ns = jb.buf, len(jb.plan)
        first.append(at)
        sl = slice(at, at + ns)
        kx = np.asarray([f[0] for f in jb.fits], np.int64)
        rs["codes_off"][sl] = codes_offs[j] + b.offsets[:ns]
        rs["out_off"][sl] = out_offs[j] // elem + b.offsets[:ns]
        rs["n"][sl] = np.asarray(b.items[:ns], np.uint32)
        rs["kexp"][sl], rs["radius"][sl], rs["mode"][sl] = kx, jb.radius, _lib.RANS_LANES
        rs["alphabet"][sl] = (1 << (kx + 1)).astype(np.uint32)
        for t in range(ns):
            kexp, level, shape, owx, bits = jb.fits[t]
            rs["framed_hi"][at + t] = bitstream.pack_frame(0, kexp, shape, level, owx, False)
            nt = int(b.items[t])
            if nt:
                cdf, enc, bucket, _ = rans_model.device_tables.get(
                    _lib.RANS_LANES, kexp, shape, owx, level, dev)
                keep.append((cdf, enc, bucket))
                rs["cdf"][at + t], rs["enc"][at + t], rs["bucket"][at + t] = (
                    cdf.data_ptr(), enc.data_ptr(), bucket.data_ptr())
                rs["K"][at + t] = rans_model.lanes_K(nt, bits)
        at += ns
    stages = rs.ctypes.data
    wsb = lib.latec_rans_encode_workspace_bytes(stages, n_all)
    ws = torch.empty(max(int(wsb), 1), dtype=torch.uint8, device=dev)
    items = rs["n"].astype(np.int64)
    cap = int(np.sum(16 + 4 * (1 + 65 * rs["n_chunks"].astype(np.int64) + items + 2)
                     + elem * items))
    cap = (cap + 15) // 16 * 16
    payload = torch.empty(cap, dtype=torch.uint8, device=dev)
    plen = torch.zeros(1, dtype=torch.int64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.latec_rans_encode(stages, n_all, codes_buf.data_ptr(), None,
                                     stats_buf.data_ptr(), out_buf.data_ptr(), elem,
                                     payload.data_ptr(), cap, plen.data_ptr(), err.data_ptr(),
                                     ws.data_ptr(), ws.numel(), _lib.stream_ptr()),
               "latec_rans_encode")
    dsz = ctypes.sizeof(_lib.RansStage) * n_all
    tail = torch.cat([plen.view(torch.uint8), err.view(torch.uint8), ws[:dsz]]).cpu().numpy()
    e = int(tail[8:12].view(np.int32)[0])
    if e:
        raise RuntimeError(f"entropy coder reported error bits {e:#x}")
    desc = (_lib.RansStage * n_all).from_buffer_copy(tail[12:12 + dsz].tobytes())
    starts, lens = [], []
    for j, jb in enumerate(jobs):
        ns = len(jb.plan)
        t0 = first[j]
        starts.append(int(desc[t0].rec_off))
        lens.append(sum(16 + 4 * int(desc[t].blob_words) + elem * int(desc[t].n_out)
                        for t in range(t0, t0 + ns)))
    if sum(lens) != int(tail[:8].view(np.int64)[0]):
        raise RuntimeError("stage records are not contiguous")
    del keep
    return payload, starts, lens


# ---------------------------------------------------------------- decode
def decompress_many(streams, *, device=None, out="numpy"):
    """Decompress a list of streams; returns the fields in order, as
    ``decompress(s, out=out)`` would. Streams may be bytes-like or CUDA
    uint8 tensors; native-mode InterpPredictor streams are decoded together,
    any other stream on its own."""
    torch = _torch()
    lib = _lib.load()
    streams = list(streams)
    if not streams:
        return []
    from .predictor import InterpPredictor

    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    sp = _lib.stream_ptr()
    # ---- headers: device prefixes in one download
    is_dev = [torch.is_tensor(s) and s.is_cuda for s in streams]
    if any(is_dev):
        pre = [s[:min(s.numel(), 4096)] for s, d in zip(streams, is_dev) if d]
        flat = torch.cat(pre).cpu().numpy().tobytes()
        at, dev_pre = 0, []
        for p in pre:
            dev_pre.append(flat[at:at + p.numel()])
            at += p.numel()
        dev_pre = iter(dev_pre)
    items = []
    for s, d in zip(streams, is_dev):
        if d:
            if s.dtype != torch.uint8 or s.dim() != 1:
                raise ValueError("a device stream must be a 1-D uint8 tensor")
            prefix, n_total = next(dev_pre), s.numel()
        else:
            mv = memoryview(s).cast("B")
            prefix, n_total = mv[:min(len(mv), 4096)].tobytes(), len(mv)
        h = Header.unpack(prefix)
        n_raw = _raw_frame_size(prefix[h.size:h.size + 13], n_total - h.size)
        batched = (h.flags & FLAG_LANES and h.flags & FLAG_INTERP and not h.flags & FLAG_RANS
                   and n_raw is not None)
        items.append((h, n_raw, n_total, bool(batched)))
    results = [None] * len(streams)
    idx = [j for j, it in enumerate(items) if it[3]]
    for j, it in enumerate(items):
        if not it[3]:
            results[j] = decompress(streams[j], device=device, out=out)
    if not idx:
        return results
    # ---- payloads: unframed into one shared buffer (host frames in one upload)
    heads = [items[j][0] for j in idx]
    n_pay = [items[j][1] for j in idx]
    pay_off = np.cumsum([0] + [-(-(n + 8) // _ALIGN) * _ALIGN for n in n_pay]).tolist()
    pay = torch.zeros(max(pay_off[-1], 1), dtype=torch.uint8, device=dev)
    host_j = [k for k, j in enumerate(idx) if not is_dev[j]]
    frames = {}
    if host_j:
        bodies = [memoryview(streams[idx[k]]).cast("B")[heads[k].size:] for k in host_j]
        boff = np.cumsum([0] + [len(b) for b in bodies]).tolist()
        pin = torch.empty(max(boff[-1], 1), dtype=torch.uint8, pin_memory=True)
        pn = pin.numpy()
        for b, a in zip(bodies, boff[:-1]):
            pn[a:a + len(b)] = np.frombuffer(b, np.uint8)
        up = pin.to(dev, non_blocking=True)
        for k, a in zip(host_j, boff[:-1]):
            frames[k] = up.data_ptr() + a
    for k, j in enumerate(idx):
        if is_dev[j]:
            frames[k] = streams[j].data_ptr() + heads[k].size
    plans, spatial, chans = [], [], []
    for h in heads:
        if h.src_dtype not in bitstream.DTYPE_CODES:
            raise KeyError(h.src_dtype)
        _check_radius(h.radius)
        sp_ = tuple(h.spatial)
        if int(h.channels) < 1:
            raise ValueError("stream has no channels")
        spatial.append(sp_)
        chans.append(int(h.channels))
        plans.append(_levels.plan_for(sp_, h.levels, h.anchor_stride, h.anchor_block))
    nss = [len(p) for p in plans]
    st0 = np.cumsum([0] + nss).tolist()
    rsz = ctypes.sizeof(_lib.Record)
    rec = torch.empty(max(st0[-1], 1) * rsz, dtype=torch.uint8, device=dev)
    tcs = torch.zeros(len(idx), dtype=torch.int64, device=dev)
    errs = torch.zeros(len(idx) + 1, dtype=torch.int32, device=dev)  # the last: the lane decoder
    for k in range(len(idx)):
        e_ptr = errs.data_ptr() + 4 * k
        _lib.check(lib.latec_unframe_raw(frames[k], n_pay[k], pay.data_ptr() + pay_off[k],
                                         e_ptr, sp), "latec_unframe_raw")
        elem = 8 if heads[k].src_dtype == 2 else 4
        _lib.check(lib.latec_parse_records(pay.data_ptr() + pay_off[k], n_pay[k], nss[k], elem, 1,
                                           rec.data_ptr() + st0[k] * rsz,
                                           tcs.data_ptr() + 8 * k, sp), "latec_parse_records")
    got = torch.cat([rec, tcs.view(torch.uint8), errs.view(torch.uint8)]).cpu().numpy()
    nrec = rec.numel()
    recs = (_lib.Record * max(st0[-1], 1)).from_buffer_copy(got[:nrec].tobytes())
    tc = got[nrec:nrec + 8 * len(idx)].view(np.int64).tolist()
    e0 = got[nrec + 8 * len(idx):].view(np.int32)
    for k in range(len(idx)):
        if e0[k] & 64:
            raise ValueError(f"stream {idx[k]}: zstd frame is corrupt")
    # ---- descriptors of every stage of every stream; one lane-decoder launch
    ch0 = np.cumsum([0] + tc).tolist()
    ranges = torch.empty(max(2 * ch0[-1], 2), dtype=torch.int64, device=dev)
    stages = (_lib.RansStage * max(st0[-1], 1))()
    keep, code_off, cat = [], [], 0
    for k, h in enumerate(heads):
        items_k = [n * chans[k] for n in plans[k].counts]
        offs = np.concatenate([[0], np.cumsum(items_k)]).astype(np.int64)
        code_off.append((cat, offs))
        word0 = pay_off[k] // 4
        for t in range(nss[k]):
            r, d = recs[st0[k] + t], stages[st0[k] + t]
            if r.status:
                raise ValueError(f"stream {idx[k]}: "
                                 + _STATUS.get(r.status, "malformed stage record"))
            f = bitstream.unpack_frame(int(r.frame))
            if r.n != items_k[t]:
                raise ValueError(f"stream {idx[k]}: stage code count mismatch")
            if not f["kexp"]:
                raise ValueError(f"stream {idx[k]}: rANS stage record has no coder window")
            if f["literal"] or (r.n == 0 and f["hlen"]) or f["hlen"] % 4:
                raise ValueError(f"stream {idx[k]}: malformed stage record")
            d.codes_off = cat + int(offs[t])
            d.n = r.n
            d.kexp, d.radius, d.mode = f["kexp"], int(h.radius), _lib.RANS_LANES
            d.alphabet = 1 << (f["kexp"] + 1)
            d.chunk0, d.n_chunks, d.K = ch0[k] + r.chunk0, r.n_chunks, r.K
            if r.n == 0:
                continue
            cdf, enc, bucket, _ = rans_model.device_tables.get(
                _lib.RANS_LANES, f["kexp"], f["shape"], f["owx"], f["level"], dev)
            keep.append((cdf, enc, bucket))
            d.cdf, d.enc, d.bucket = cdf.data_ptr(), enc.data_ptr(), bucket.data_ptr()
            d.blob_off = word0 + r.blob // 4
            d.blob_words = f["hlen"] // 4
        if tc[k]:
            _lib.check(lib.latec_chunk_ranges(pay.data_ptr() + pay_off[k],
                                              rec.data_ptr() + st0[k] * rsz, nss[k],
                                              ranges.data_ptr() + 16 * ch0[k],
                                              errs.data_ptr() + 4 * k, sp), "latec_chunk_ranges")
            ranges[2 * ch0[k]:2 * ch0[k + 1]] += word0  # positions in the shared buffer
        cat += int(offs[-1])
    codes = torch.empty(max(cat, 1), dtype=torch.int16, device=dev)
    n_all = st0[-1]
    ws = torch.empty(int(lib.latec_rans_decode_workspace_bytes(n_all)), dtype=torch.uint8,
                     device=dev)
    _lib.check(lib.latec_rans_decode(stages, n_all, ch0[-1], pay.data_ptr(),
                                     ranges.data_ptr() if ch0[-1] else None, None,
                                     codes.data_ptr(), errs.data_ptr() + 4 * len(idx),
                                     ws.data_ptr(), ws.numel(), sp), "latec_rans_decode")
    # ---- every field rebuilt by the stage kernels: stage index by stage
    # index, one launch per kernel class over all fields
    canv = []
    dj = (_lib.DecodeJob * len(heads))()
    hold = []
    for k, h in enumerate(heads):
        c = chans[k]
        pred = InterpPredictor("cubic" if h.flags & FLAG_CUBIC else "linear", h.levels,
                               h.anchor_stride, h.anchor_block)
        end_mode = (h.flags >> END_MODE_SHIFT) & END_MODE_MAX
        ebs = _levels.stage_ebs(spatial[k], h.levels, h.anchor_stride, h.anchor_block, h.eb,
                                h.eb_ratio)
        ns = nss[k]
        prm = _qparams(h.src_dtype, c, h.radius, pred.order, h.interp_center, end_mode,
                       h.src_dtype == 0)
        ft = torch.float64 if h.src_dtype == 2 else torch.float32
        recon = torch.empty((c,) + spatial[k], dtype=ft, device=dev)  # every point decoded
        eb_arr = (ctypes.c_double * ns)(*[float(e) for e in ebs])
        out_at = (ctypes.c_uint64 * ns)(*[recs[st0[k] + t].out_at for t in range(ns)])
        n_out = (ctypes.c_uint32 * ns)(*[recs[st0[k] + t].n_out for t in range(ns)])
        d = dj[k]
        d.plan, d.prm = plans[k].handle, prm
        d.stage_eb, d.out_off, d.n_out = (ctypes.addressof(eb_arr), ctypes.addressof(out_at),
                                          ctypes.addressof(n_out))
        d.codes = codes.data_ptr() + 2 * code_off[k][0]
        d.outliers = pay.data_ptr() + pay_off[k]
        d.recon, d.err = recon.data_ptr(), errs.data_ptr() + 4 * k
        hold.append((eb_arr, out_at, n_out))
        canv.append(recon)
    tb = int(lib.latec_decode_many_table_bytes(dj, len(heads)))
    if not tb:
        raise ValueError("latec_decode_many_table_bytes: invalid job")
    table = torch.empty(tb, dtype=torch.uint8, device=dev)
    _lib.check(lib.latec_decode_stages_many(dj, len(heads), table.data_ptr(), tb, sp),
               "latec_decode_stages_many")
    del hold
    e = errs.cpu().numpy()  # one download: every stream's error word
    del keep
    lane = int(e[-1])
    for k in range(len(idx)):
        ek = int(e[k]) | lane
        if ek & 1:
            raise ValueError(f"stream {idx[k]}: outlier count mismatch")
        if ek & (4 | 8 | 128):
            raise ValueError(f"stream {idx[k]}: trailing data in rANS payload")
        if ek & 16:
            raise ValueError(f"stream {idx[k]}: malformed rANS payload")
        if ek:
            raise ValueError(f"stream {idx[k]}: malformed stream (error bits {ek:#x})")
    for k, j in enumerate(idx):
        results[j] = _finalize(canv[k], heads[k].src_dtype, chans[k], as_numpy=(out == "numpy"))
    return results
