"""Test-only stand-in for the ``zstandard`` package, used when importing the
reference LATEC package to generate golden vectors.

Only the calls the reference makes are provided: ``ZstdCompressor(level).compress``
and ``ZstdDecompressor().decompress``, both over the system ``libzstd.so.1``.
"""

import ctypes
import ctypes.util

_lib = ctypes.CDLL(ctypes.util.find_library("zstd") or "libzstd.so.1")
_lib.ZSTD_compressBound.restype = ctypes.c_size_t
_lib.ZSTD_compressBound.argtypes = [ctypes.c_size_t]
_lib.ZSTD_compress.restype = ctypes.c_size_t
_lib.ZSTD_compress.argtypes = [
    ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
_lib.ZSTD_decompress.restype = ctypes.c_size_t
_lib.ZSTD_decompress.argtypes = [
    ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
_lib.ZSTD_getFrameContentSize.restype = ctypes.c_ulonglong
_lib.ZSTD_getFrameContentSize.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
_lib.ZSTD_isError.restype = ctypes.c_uint
_lib.ZSTD_isError.argtypes = [ctypes.c_size_t]


class ZstdError(Exception):
    pass


class ZstdCompressor:
    def __init__(self, level=3):
        self.level = int(level)

    def compress(self, data):
        data = bytes(data)
        cap = _lib.ZSTD_compressBound(len(data))
        out = ctypes.create_string_buffer(cap)
        n = _lib.ZSTD_compress(out, cap, data, len(data), self.level)
        if _lib.ZSTD_isError(n):
            raise ZstdError("compress failed")
        return out.raw[:n]


class ZstdDecompressor:
    def decompress(self, data):
        data = bytes(data)
        size = _lib.ZSTD_getFrameContentSize(data, len(data))
        if size >= (1 << 63):
            raise ZstdError("could not determine content size in frame header")
        out = ctypes.create_string_buffer(max(int(size), 1))
        n = _lib.ZSTD_decompress(out, int(size), data, len(data))
        if _lib.ZSTD_isError(n):
            raise ZstdError("decompress failed")
        return out.raw[:n]
