"""Oracle restatement of the closed-loop plain codec and its container.

Test infrastructure only (see ``oracle/__init__.py``). Follows
``latec/codec.py:45-322,384-524`` (fast tune) and ``latec/bitstream.py``.

Two entropy modes, selected by the container flag ``FLAG_LANES``:

* ``"compat"`` -- the reference's stream: stage-constant rANS through the
  constriction-compatible stack coder, the literal-zstd back end when it wins
  (``latec/bitstream.py:203-219``), and a level-``zstd_level`` zstd frame
  around the payload.
* ``"native"`` -- the CUDA library's stream: the same stage records, but each
  rANS blob is the 32-lane interleaved coder of ``oracle/ans.c`` with the
  reference's own 24-bit tables, the stage model fitted with exact fixed-point
  costs (``rans_model.fit_const_native``), no literal stages, and the payload
  stored in a zstd frame of raw blocks (decodable by any zstd decoder).

float64 input (new; the reference raises on it) uses dtype id 2, keeps the
reconstruction, the predictions and the outliers in float64 and checks the
bound in float64.
"""

from __future__ import annotations

import ctypes
import ctypes.util
import math
import struct

import numpy as np

from . import ans, interp, levels, quant, rans_model

MAGIC = b"LATEC001"
VERSION = 4
FLAG_INTERP = 1 << 3
FLAG_CUBIC = 1 << 4
FLAG_LANES = 1 << 11
END_MODE_SHIFT = 9
HEADER_FMT = "<8sHHIIBBBBIHhddd16sd"
HEADER_SIZE = struct.calcsize(HEADER_FMT)
DTYPE_IDS = {np.dtype(np.uint8): 0, np.dtype(np.float32): 1, np.dtype(np.float64): 2}
_HLEN_BITS, _KEXP_SHIFT, _SHAPE_SHIFT, _LEVEL_SHIFT, _OWX_SHIFT, _LIT_SHIFT = 45, 45, 49, 54, 60, 63
_LITERAL_MIN = 1 << 12
_SCOUT_SLACK = 0.85
LANES_KMIN, LANES_KMAX, LANES_BITS_PER_WARP = 16, 8192, 131072


# ---------------------------------------------------------------- zstd

class _Zstd:
    def __init__(self):
        L = ctypes.CDLL(ctypes.util.find_library("zstd") or "libzstd.so.1")
        L.ZSTD_compressBound.restype = ctypes.c_size_t
        L.ZSTD_compressBound.argtypes = [ctypes.c_size_t]
        L.ZSTD_compress.restype = ctypes.c_size_t
        L.ZSTD_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                    ctypes.c_size_t, ctypes.c_int]
        L.ZSTD_decompress.restype = ctypes.c_size_t
        L.ZSTD_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                      ctypes.c_size_t]
        L.ZSTD_getFrameContentSize.restype = ctypes.c_ulonglong
        L.ZSTD_getFrameContentSize.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        L.ZSTD_isError.restype = ctypes.c_uint
        L.ZSTD_isError.argtypes = [ctypes.c_size_t]
        self.L = L

    def compress(self, data: bytes, level: int) -> bytes:
        cap = self.L.ZSTD_compressBound(len(data))
        out = ctypes.create_string_buffer(cap)
        n = self.L.ZSTD_compress(out, cap, data, len(data), level)
        if self.L.ZSTD_isError(n):
            raise ValueError("zstd compress failed")
        return out.raw[:n]

    def decompress(self, data: bytes) -> bytes:
        size = self.L.ZSTD_getFrameContentSize(data, len(data))
        if size >= (1 << 63):
            raise ValueError("zstd frame without content size")
        out = ctypes.create_string_buffer(max(int(size), 1))
        n = self.L.ZSTD_decompress(out, int(size), data, len(data))
        if self.L.ZSTD_isError(n) or n != size:
            raise ValueError("zstd decompress failed")
        return out.raw[:n]


_zstd = None


def zstd():
    global _zstd
    if _zstd is None:
        _zstd = _Zstd()
    return _zstd


def raw_zstd_frame(payload: bytes) -> bytes:
    """A single-segment zstd frame of raw (stored) blocks, content size in the
    header (zstd format spec: frame header descriptor 0xE0, 8-byte FCS, blocks
    of at most 128 KiB with 3-byte headers ``last | type 0 << 1 | size << 3``)."""
    out = [struct.pack("<IBQ", 0xFD2FB528, 0xE0, len(payload))]
    blk = 1 << 17
    n = len(payload)
    if n == 0:
        out.append((1).to_bytes(3, "little"))
    for a in range(0, n, blk):
        size = min(blk, n - a)
        last = 1 if a + size >= n else 0
        out.append((last | (size << 3)).to_bytes(3, "little"))
        out.append(payload[a:a + size])
    return b"".join(out)


# ---------------------------------------------------------------- header

def pack_header(h: dict) -> bytes:
    """``latec/bitstream.py:78-103``."""
    fixed = struct.pack(HEADER_FMT, MAGIC, VERSION, h["flags"], h["channels"], h["src_dtype"],
                        h["levels"], h["anchor_stride"], h["anchor_block"], h["interp_center"],
                        h["radius"], h.get("max_radius", 0), h.get("agg_level", -1), h["eb"],
                        h["vmin"], h["vmax"], h.get("ckpt_hash", b"\0" * 16), h["eb_ratio"])
    sp = h["spatial"]
    return fixed + struct.pack(f"<B{len(sp)}I", len(sp), *sp)


def unpack_header(buf: bytes) -> dict:
    """``latec/bitstream.py:105-152``."""
    (magic, version, flags, channels, src_dtype, lv, stride, block, center, radius, max_radius,
     agg, eb, vmin, vmax, ckpt, ratio) = struct.unpack_from(HEADER_FMT, buf, 0)
    if magic != MAGIC:
        raise ValueError("bad magic")
    if version != VERSION:
        raise ValueError("unsupported version")
    (nd,) = struct.unpack_from("<B", buf, HEADER_SIZE)
    if not nd:
        raise ValueError("stream spatial shape is empty")
    spatial = struct.unpack_from(f"<{nd}I", buf, HEADER_SIZE + 1)
    return dict(flags=flags, channels=channels, src_dtype=src_dtype, levels=lv,
                anchor_stride=stride, anchor_block=block, interp_center=center, radius=radius,
                max_radius=max_radius, agg_level=agg, eb=eb, vmin=vmin, vmax=vmax,
                ckpt_hash=ckpt, eb_ratio=ratio, spatial=tuple(spatial),
                body_offset=HEADER_SIZE + 1 + 4 * nd)


def framed(hlen, kexp, shape, level=0, owx=0, literal=False):
    """``latec/bitstream.py:260-285``."""
    if hlen >= 1 << _HLEN_BITS:
        raise ValueError("stage entropy blob is too large to frame")
    return (hlen | (kexp << _KEXP_SHIFT) | (shape << _SHAPE_SHIFT) | (level << _LEVEL_SHIFT)
            | (owx << _OWX_SHIFT) | (int(literal) << _LIT_SHIFT))


def unframe(word):
    return dict(hlen=word & ((1 << _HLEN_BITS) - 1), kexp=(word >> _KEXP_SHIFT) & 15,
                shape=(word >> _SHAPE_SHIFT) & 31, level=(word >> _LEVEL_SHIFT) & 63,
                owx=(word >> _OWX_SHIFT) & 7, literal=bool((word >> _LIT_SHIFT) & 1))


def lanes_K(n, model_bits):
    """Symbols per lane of the native coder for a stage of ``n`` codes whose
    fitted model prices it at ``model_bits``: as many 32-lane chunks as keep the
    64-bit final states under ~1/64 of the stage's bits, within
    ``[LANES_KMIN, LANES_KMAX]`` symbols per lane."""
    lo = -(-n // (32 * LANES_KMAX))
    hi = -(-n // (32 * LANES_KMIN))
    warps = max(lo, min(hi, max(1, int(math.floor(model_bits / LANES_BITS_PER_WARP)))))
    return -(-n // (32 * warps))


def literal_dtype(kexp):
    return np.dtype(np.uint8 if kexp <= 7 else np.uint16)


def pack_stage(codes, outliers, radius, mode, zstd_level=9):
    """Stage record; ``latec/bitstream.py:178-243`` (stage-constant path)."""
    codes = np.asarray(codes, np.uint32)
    kexp = rans_model.choose_kexp(codes, radius)
    if mode == "native" and len(codes):
        counts = np.bincount(rans_model.narrow(codes, radius, kexp), minlength=2 << kexp)
        level, shape, owx, bits = rans_model.fit_const_native(counts, len(codes), kexp)
    else:
        level, shape, owx, bits = rans_model.choose_const_level(codes, radius, kexp)
    literal = False
    blob = None
    syms = rans_model.narrow(codes, radius, kexp) if len(codes) else np.zeros(0, np.int64)
    if mode == "compat" and len(codes) >= _LITERAL_MIN:
        lit = syms.astype(literal_dtype(kexp)).tobytes()
        scout = zstd().compress(lit, 1)
        if len(scout) * _SCOUT_SLACK < bits / 8.0:
            b = zstd().compress(lit, zstd_level)
            if len(b) * 8.0 < bits:
                blob, literal = b, True
    if blob is None:
        if len(codes) == 0:
            blob = b""
        elif mode == "compat":
            cdf = ans.wire_cdfs(rans_model.build_cdfs(kexp, shape, owx=owx)[level:level + 1])
            blob = ans.stack_encode(syms, cdf)
        else:
            cdf = rans_model.build_cdfs(kexp, shape, owx=owx)[level]
            blob = ans.lanes_encode(syms, cdf, lanes_K(len(codes), bits))
    rec = (struct.pack("<IQ", len(codes), framed(len(blob), kexp, shape, level, owx, literal))
           + blob + struct.pack("<I", len(outliers)) + np.asarray(outliers).tobytes())
    return rec, dict(kexp=kexp, level=level, shape=shape, owx=owx, model_bits=bits,
                     literal=literal, blob_bytes=len(blob))


def unpack_stage(buf, off, radius, mode, out_dtype):
    """``latec/bitstream.py:288-344`` (stage-constant path)."""
    n, word = struct.unpack_from("<IQ", buf, off)
    f = unframe(word)
    off += 12
    blob = buf[off:off + f["hlen"]]
    if not f["kexp"]:
        raise ValueError("rANS stage record has no coder window")
    if f["literal"]:
        syms = np.frombuffer(zstd().decompress(blob), literal_dtype(f["kexp"]), count=n)
    elif n == 0:
        if blob:
            raise ValueError("non-empty rANS blob for an empty stage")
        syms = np.zeros(0, np.int64)
    elif mode == "compat":
        cdf = ans.wire_cdfs(rans_model.build_cdfs(f["kexp"], f["shape"], owx=f["owx"])
                            [f["level"]:f["level"] + 1])
        syms = ans.stack_decode(blob, n, cdf)
    else:
        cdf = rans_model.build_cdfs(f["kexp"], f["shape"], owx=f["owx"])[f["level"]]
        syms = ans.lanes_decode(blob, n, cdf)
    codes = rans_model.widen(syms, radius, f["kexp"])
    off += f["hlen"]
    (n_out,) = struct.unpack_from("<I", buf, off)
    off += 4
    isz = np.dtype(out_dtype).itemsize
    outliers = np.frombuffer(buf, out_dtype, count=n_out, offset=off).copy()
    off += isz * n_out
    return codes, outliers, off


# ---------------------------------------------------------------- codec

def _normalise(img):
    """``latec/codec.py:77-91`` plus float64 (dtype id 2)."""
    img = np.asarray(img)
    is_image = img.ndim <= 2 or (img.ndim == 3 and img.shape[-1] in (1, 3))
    f64 = img.dtype == np.float64
    ft = np.float64 if f64 else np.float32
    if is_image:
        if img.ndim == 2:
            img = img[..., None]
        spatial, c = img.shape[:-1], img.shape[-1]
        fimg = np.asarray(img, ft)
    else:
        spatial, c = img.shape, 1
        fimg = np.asarray(img, ft)[..., None]
    src = DTYPE_IDS[np.dtype(img.dtype)]
    return fimg, tuple(spatial), c, src


def compress(img, eb, order="cubic", levels_=4, anchor_stride=16, anchor_block=1,
             radius=1 << 15, zstd_level=9, eb_ratio=None, center=None, end_mode=None,
             mode="native"):
    """Fast-tune encode; returns ``(stream, stats)`` like ``latec/codec.py:45-285``."""
    fimg, spatial, c, src = _normalise(img)
    if len(spatial) < 1:
        raise ValueError("shape must have at least one axis")
    vmin, vmax = float(fimg.min()), float(fimg.max())
    if vmax <= vmin:
        vmax = vmin + 1.0
    nd = len(spatial)
    if center is None:
        center = 1 if nd >= 4 else 0
    if end_mode is None:
        end_mode = interp.END_QUAD
    ratio = 0.9 if eb_ratio is None else eb_ratio
    field = np.moveaxis(fimg, -1, 0)
    ebs = levels.stage_ebs(spatial, levels_, anchor_stride, anchor_block, eb, ratio)
    recon = np.zeros_like(field)
    flat_field = field.reshape(c, -1)
    flat_recon = recon.reshape(c, -1)
    parts, recs = [], []
    for t, (mask, s, axes) in enumerate(levels.iter_plan(spatial, levels_, anchor_stride,
                                                         anchor_block)):
        idx = np.flatnonzero(mask)
        n = len(idx)
        if n == 0:
            rec, info = pack_stage(np.zeros(0, np.uint32), np.zeros(0, field.dtype), radius, mode,
                                   zstd_level)
            parts.append(rec)
            recs.append(dict(info, codes=np.zeros(0, np.uint32), outliers=np.zeros(0)))
            continue
        if t == 0:
            pred = np.zeros((c, n), field.dtype)
        else:
            pred = interp.predict(recon, s, axes, idx, order, center, end_mode)
        vals = flat_field[:, idx]
        codes, outl = quant.quantize(vals, pred, ebs[t], radius, round_output=(src == 0))
        flat_recon[:, idx] = quant.dequantize(pred, codes, outl, ebs[t], radius).reshape(c, n)
        rec, info = pack_stage(codes, outl, radius, mode, zstd_level)
        parts.append(rec)
        recs.append(dict(info, codes=codes, outliers=outl))
    payload = b"".join(parts)
    flags = FLAG_INTERP | (FLAG_CUBIC if order == "cubic" else 0) | (end_mode << END_MODE_SHIFT)
    if mode == "native":
        flags |= FLAG_LANES
    header = pack_header(dict(flags=flags, channels=c, src_dtype=src, levels=levels_,
                              anchor_stride=anchor_stride, anchor_block=anchor_block,
                              interp_center=center, radius=radius, eb=float(eb), vmin=vmin,
                              vmax=vmax, eb_ratio=ratio, spatial=spatial))
    body = raw_zstd_frame(payload) if mode == "native" else zstd().compress(payload, zstd_level)
    stream = header + body
    out = np.moveaxis(recon, 0, -1)
    if src == 0:
        out = np.clip(np.rint(out), 0, 255).astype(np.uint8)
    if c == 1:
        out = out[..., 0]
    return stream, dict(recon=out, stages=recs, payload=payload, center=center,
                        end_mode=end_mode, eb_ratio=ratio)


END_MODE_MAX = 3


def tune_sweep(img, eb, tune="size", order="cubic", levels_=4, anchor_stride=16,
               anchor_block=1, radius=1 << 15, zstd_level=9, tune_size_slack=1.05,
               mode="compat"):
    """The encoder's sequential tune sweep, ``latec/codec.py:171-262``: the base
    candidate, then every end mode at the first eb ratio, then every (eb ratio,
    center) at the smallest stream's end mode; ``"size"`` keeps the smallest
    stream, ``"rd"`` the lowest reconstruction SSE within ``tune_size_slack``
    of it (ties broken by size, ratio, center, end mode). Returns
    ``(stream, stats, (ratio, center, end_mode), n_candidates)``."""
    fimg, spatial, c, src = _normalise(img)
    nd = len(spatial)
    base_center, base_end = (1 if nd >= 4 else 0), interp.END_QUAD
    if tune not in ("fast", "size", "rd"):
        raise ValueError("tune must be 'fast', 'size', or 'rd'")
    sweep = tune != "fast"
    ratio_cands = [1.0, 0.9, 0.8, 0.7] if sweep else [0.9]
    center_cands = [base_center] + ([x for x in (0, 1, 2) if x != base_center] if sweep else [])
    field = np.asarray(img)
    cands, seen = [], set()

    def run_once(ratio, center, end_mode):
        if (ratio, center, end_mode) in seen:
            return
        seen.add((ratio, center, end_mode))
        stream, st = compress(img, eb, order, levels_, anchor_stride, anchor_block, radius,
                              zstd_level, eb_ratio=ratio, center=center, end_mode=end_mode,
                              mode=mode)
        # reconstruction error: float32 (source-precision) differences, squared in float64
        d = (np.asarray(field, fimg.dtype) - np.asarray(st["recon"], fimg.dtype))
        sse = float(np.sum(np.square(d.astype(np.float64))))
        cands.append((len(stream), sse, ratio, center, end_mode, stream, st))

    run_once(ratio_cands[0], base_center, base_end)
    chosen_end = base_end
    if sweep:
        for em in range(END_MODE_MAX + 1):
            run_once(ratio_cands[0], base_center, em)
        chosen_end = min(cands, key=lambda x: (x[0], x[1]))[4]
    for ratio in ratio_cands:
        for center in center_cands:
            run_once(ratio, center, chosen_end)
    if tune == "rd" and len(cands) > 1:
        limit = min(x[0] for x in cands) * tune_size_slack
        best = min((x for x in cands if x[0] <= limit), key=lambda x: (x[1], x[0], x[2], x[3], x[4]))
    else:
        best = min(cands, key=lambda x: (x[0], x[1], x[2], x[3], x[4]))
    return best[5], best[6], (best[2], best[3], best[4]), len(cands)


def decompress(stream: bytes):
    """``latec/codec.py:288-322,462-524``."""
    h = unpack_header(stream)
    payload = zstd().decompress(stream[h["body_offset"]:])
    mode = "native" if h["flags"] & FLAG_LANES else "compat"
    order = "cubic" if h["flags"] & FLAG_CUBIC else "linear"
    end_mode = (h["flags"] >> END_MODE_SHIFT) & 3
    spatial, c = h["spatial"], h["channels"]
    ft = np.float64 if h["src_dtype"] == 2 else np.float32
    ebs = levels.stage_ebs(spatial, h["levels"], h["anchor_stride"], h["anchor_block"], h["eb"],
                           h["eb_ratio"])
    recon = np.zeros((c, *spatial), ft)
    flat_recon = recon.reshape(c, -1)
    off = 0
    for t, (mask, s, axes) in enumerate(levels.iter_plan(spatial, h["levels"], h["anchor_stride"],
                                                         h["anchor_block"])):
        idx = np.flatnonzero(mask)
        codes, outl, off = unpack_stage(payload, off, h["radius"], mode, ft)
        if len(idx) == 0:
            continue
        if len(codes) != c * len(idx):
            raise ValueError("stage code count mismatch")
        if t == 0:
            pred = np.zeros((c, len(idx)), ft)
        else:
            pred = interp.predict(recon, s, axes, idx, order, h["interp_center"], end_mode)
        flat_recon[:, idx] = quant.dequantize(pred, codes, outl, ebs[t], h["radius"]).reshape(
            c, len(idx))
    out = np.moveaxis(recon, 0, -1)
    if h["src_dtype"] == 0:
        out = np.clip(np.rint(out), 0, 255).astype(np.uint8)
    if c == 1:
        out = out[..., 0]
    return out
