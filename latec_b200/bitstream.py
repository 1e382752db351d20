"""LATEC001 container (reference ``latec/bitstream.py``), byte-compatible.

File = fixed little-endian header ``<8sHHIIBBBBIHhddd16sd`` + ``[ndim u8]`` +
``ndim x u32`` + one zstd frame holding the stage payload. Each stage record is
``u32 n_codes | u64 frame | blob | u32 n_outliers | outliers``, the frame word
packing ``len 45b | kexp 4b | shape 5b | level 6b | owx 3b | lit 1b``.

Two additions, both flagged in the header so the reference layout is
unchanged otherwise: ``FLAG_LANES`` marks rANS blobs written by the native
32-lane interleaved coder, and dtype id 2 marks float64 sources (outliers
stored as float64).
"""

from __future__ import annotations

import ctypes
import ctypes.util
import struct
from dataclasses import dataclass

import numpy as np

MAGIC = b"LATEC001"
VERSION = 4

FLAG_MOCK = 1 << 0
FLAG_GRAY = 1 << 1
FLAG_INTERP = 1 << 3
FLAG_CUBIC = 1 << 4
FLAG_NOTILE = 1 << 5
FLAG_RANS = 1 << 6
FLAG_END_QUAD = 1 << 9
FLAG_END_EXTRAP = 1 << 10
END_MODE_SHIFT = 9
FLAG_LANES = 1 << 11  # stage blobs use the native multi-lane rANS coder

_HEADER_FMT = "<8sHHIIBBBBIHhddd16sd"
_HEADER_SIZE = struct.calcsize(_HEADER_FMT)

DTYPE_CODES = {0: np.uint8, 1: np.float32, 2: np.float64}
DTYPE_IDS = {np.dtype(np.uint8): 0, np.dtype(np.float32): 1, np.dtype(np.float64): 2}

_HLEN_BITS = 45
_KEXP_SHIFT = 45
_SHAPE_SHIFT = 49
_LEVEL_SHIFT = 54
_OWX_SHIFT = 60
_LIT_SHIFT = 63


@dataclass
class Header:
    """``latec/bitstream.py:58-152``."""

    channels: int
    src_dtype: int
    spatial: tuple
    eb: float
    levels: int
    anchor_stride: int
    anchor_block: int
    radius: int
    max_radius: int
    agg_level: int
    vmin: float
    vmax: float
    ckpt_hash: bytes = b"\0" * 16
    flags: int = 0
    interp_center: int = 0
    eb_ratio: float = 1.0
    version: int = VERSION

    def pack(self) -> bytes:
        fixed = struct.pack(
            _HEADER_FMT, MAGIC, self.version, self.flags, self.channels, self.src_dtype,
            self.levels, self.anchor_stride, self.anchor_block, self.interp_center, self.radius,
            self.max_radius, self.agg_level, self.eb, self.vmin, self.vmax, self.ckpt_hash,
            self.eb_ratio)
        if not self.spatial or len(self.spatial) > 255:
            raise ValueError("spatial shape must contain 1..255 dimensions")
        return fixed + struct.pack(f"<B{len(self.spatial)}I", len(self.spatial), *self.spatial)

    @classmethod
    def unpack(cls, buf) -> "Header":
        if len(buf) < _HEADER_SIZE + 1:
            raise ValueError("not a LATEC stream (truncated header)")
        (magic, version, flags, channels, src_dtype, levels, anchor_stride, anchor_block,
         interp_center, radius, max_radius, agg_level, eb, vmin, vmax, ckpt_hash,
         eb_ratio) = struct.unpack_from(_HEADER_FMT, buf, 0)
        if magic != MAGIC:
            raise ValueError(f"not a LATEC stream (bad magic {magic!r})")
        if version != VERSION:
            raise ValueError(f"unsupported version {version}")
        (ndim,) = struct.unpack_from("<B", buf, _HEADER_SIZE)
        if not ndim:
            raise ValueError("stream spatial shape is empty")
        if len(buf) < _HEADER_SIZE + 1 + 4 * ndim:
            raise ValueError("not a LATEC stream (truncated header)")
        spatial = struct.unpack_from(f"<{ndim}I", buf, _HEADER_SIZE + 1)
        return cls(channels=channels, src_dtype=src_dtype, spatial=tuple(spatial), eb=eb,
                   levels=levels, anchor_stride=anchor_stride, anchor_block=anchor_block,
                   radius=radius, max_radius=max_radius, agg_level=agg_level, vmin=vmin,
                   vmax=vmax, ckpt_hash=ckpt_hash, flags=flags, interp_center=interp_center,
                   eb_ratio=eb_ratio, version=version)

    @property
    def size(self) -> int:
        return _HEADER_SIZE + 1 + 4 * len(self.spatial)


def pack_frame(hlen, kexp, shape, level=0, owx=0, literal=False) -> int:
    """Stage frame word (``latec/bitstream.py:260-285``)."""
    if hlen >= 1 << _HLEN_BITS:
        raise ValueError("stage entropy blob is too large to frame")
    if not 0 <= int(kexp) < 16:
        raise ValueError("rANS coder window does not fit the stage frame")
    if not 0 <= int(shape) < 32:
        raise ValueError("rANS shape id does not fit the stage frame")
    if not 0 <= int(level) < 64:
        raise ValueError("rANS scale level does not fit the stage frame")
    if not 0 <= int(owx) < 8:
        raise ValueError("rANS outlier weight does not fit the stage frame")
    return (int(hlen) | (int(kexp) << _KEXP_SHIFT) | (int(shape) << _SHAPE_SHIFT)
            | (int(level) << _LEVEL_SHIFT) | (int(owx) << _OWX_SHIFT)
            | (int(bool(literal)) << _LIT_SHIFT))


def unpack_frame(word: int) -> dict:
    return dict(hlen=word & ((1 << _HLEN_BITS) - 1), kexp=(word >> _KEXP_SHIFT) & 15,
                shape=(word >> _SHAPE_SHIFT) & 31, level=(word >> _LEVEL_SHIFT) & 63,
                owx=(word >> _OWX_SHIFT) & 7, literal=bool((word >> _LIT_SHIFT) & 1))


# ------------------------------------------------------------------ zstd

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

    def compress(self, data, level: int) -> bytes:
        data = memoryview(data).cast("B")
        src = np.frombuffer(data, np.uint8)
        cap = self.L.ZSTD_compressBound(len(src))
        out = np.empty(cap, np.uint8)
        n = self.L.ZSTD_compress(out.ctypes.data, cap, src.ctypes.data, len(src), int(level))
        if self.L.ZSTD_isError(n):
            raise ValueError("zstd compression failed")
        return out[:n].tobytes()

    def decompress_into(self, data) -> np.ndarray:
        src = np.frombuffer(memoryview(data).cast("B"), np.uint8)
        size = self.L.ZSTD_getFrameContentSize(src.ctypes.data, len(src))
        if size >= (1 << 63):
            raise ValueError("could not determine content size in frame header")
        out = np.empty(max(int(size), 1), np.uint8)
        n = self.L.ZSTD_decompress(out.ctypes.data, int(size), src.ctypes.data, len(src))
        if self.L.ZSTD_isError(n) or n != size:
            raise ValueError("zstd frame is corrupt")
        return out[:n]


_zstd = None


def zstd() -> _Zstd:
    global _zstd
    if _zstd is None:
        _zstd = _Zstd()
    return _zstd


_RAW_BLOCK = 1 << 17


def raw_zstd_frame(payload: np.ndarray) -> np.ndarray:
    """Wrap ``payload`` (uint8) in a single-segment zstd frame of raw blocks
    (zstd format: magic, descriptor 0xE0 = 8-byte content size + single
    segment, then blocks with 3-byte headers ``last | raw << 1 | size << 3``).
    Any zstd decoder reads it; writing it is a strided copy."""
    payload = np.ascontiguousarray(payload, np.uint8).reshape(-1)
    n = len(payload)
    nblk = max(1, -(-n // _RAW_BLOCK))
    out = np.empty(13 + 3 * nblk + n, np.uint8)
    out[:13] = np.frombuffer(struct.pack("<IBQ", 0xFD2FB528, 0xE0, n), np.uint8)
    full = n // _RAW_BLOCK
    if full:
        body = out[13:13 + full * (_RAW_BLOCK + 3)].reshape(full, _RAW_BLOCK + 3)
        hdr = ((_RAW_BLOCK << 3)).to_bytes(3, "little")
        body[:, :3] = np.frombuffer(hdr, np.uint8)
        body[:, 3:] = payload[:full * _RAW_BLOCK].reshape(full, _RAW_BLOCK)
    rest = n - full * _RAW_BLOCK
    if rest or n == 0:
        a = 13 + full * (_RAW_BLOCK + 3)
        out[a:a + 3] = np.frombuffer((1 | (rest << 3)).to_bytes(3, "little"), np.uint8)
        out[a + 3:a + 3 + rest] = payload[full * _RAW_BLOCK:]
    else:  # last full block carries the last-block bit
        a = 13 + (full - 1) * (_RAW_BLOCK + 3)
        out[a] |= 1
    return out


class PayloadReader:
    """Random access to the stage payload, either a plain host array or the
    payload inside a zstd frame of raw blocks (payload byte ``p`` sits at frame
    offset ``13 + 3 * (p // 128 KiB + 1) + p``), without unframing it on the host."""

    def __init__(self, data: np.ndarray, n: int, framed: bool):
        self.data, self.n, self.framed = data, int(n), framed

    def __len__(self):
        return self.n

    def _idx(self, p, k):
        idx = np.arange(p, p + k, dtype=np.int64)
        if self.framed:
            idx = 13 + 3 * (idx // _RAW_BLOCK + 1) + idx
        return idx

    def take(self, p: int, k: int) -> np.ndarray:
        if p < 0 or p + k > self.n:
            raise ValueError("truncated stage record")
        if not self.framed:
            return self.data[p:p + k]
        return self.data[self._idx(p, k)]

    def u32s(self, p: int, count: int) -> np.ndarray:
        return np.ascontiguousarray(self.take(p, 4 * count)).view("<u4")

    def unpack(self, fmt: str, p: int):
        return struct.unpack(fmt, self.take(p, struct.calcsize(fmt)).tobytes())


def raw_frame_size(body: np.ndarray):
    """Payload size if ``body`` is exactly a single-segment zstd frame of raw
    blocks in the layout ``raw_zstd_frame`` writes, else None."""
    if len(body) < 13 or bytes(body[:5]) != struct.pack("<IB", 0xFD2FB528, 0xE0):
        return None
    (n,) = struct.unpack_from("<Q", body, 5)
    nblk = max(1, -(-n // _RAW_BLOCK))
    if len(body) != 13 + 3 * nblk + n:
        return None
    starts = 13 + np.arange(nblk, dtype=np.int64) * (_RAW_BLOCK + 3)
    hdr = (body[starts].astype(np.uint32) | (body[starts + 1].astype(np.uint32) << 8)
           | (body[starts + 2].astype(np.uint32) << 16))
    sizes = np.full(nblk, _RAW_BLOCK, np.uint32)
    sizes[-1] = n - (nblk - 1) * _RAW_BLOCK
    want = sizes << 3
    want[-1] |= 1
    return int(n) if np.array_equal(hdr, want) else None


def read_body(data) -> np.ndarray:
    """Decode the zstd frame after the header into the payload bytes. Frames of
    raw blocks (the native writer's) are unpacked with a strided copy; any
    other frame goes through libzstd."""
    src = np.frombuffer(memoryview(data).cast("B"), np.uint8)
    if len(src) >= 13 and bytes(src[:5]) == struct.pack("<IB", 0xFD2FB528, 0xE0):
        (n,) = struct.unpack_from("<Q", src, 5)
        full, rest = divmod(n, _RAW_BLOCK)
        nblk = max(1, -(-n // _RAW_BLOCK))
        if len(src) == 13 + 3 * nblk + n:
            ok = True
            if full:
                body = src[13:13 + full * (_RAW_BLOCK + 3)].reshape(full, _RAW_BLOCK + 3)
                hdr = body[:, 0].astype(np.uint32) | (body[:, 1].astype(np.uint32) << 8) | (
                    body[:, 2].astype(np.uint32) << 16)
                want = np.full(full, _RAW_BLOCK << 3, np.uint32)
                if not rest and n:
                    want[-1] |= 1
                ok = bool(np.array_equal(hdr, want))
            if ok:
                out = np.empty(n, np.uint8)
                if full:
                    out[:full * _RAW_BLOCK] = body[:, 3:].reshape(-1)
                if rest:
                    a = 13 + full * (_RAW_BLOCK + 3)
                    out[full * _RAW_BLOCK:] = src[a + 3:a + 3 + rest]
                return out
    return zstd().decompress_into(src)
