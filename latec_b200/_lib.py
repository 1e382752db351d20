"""ctypes binding of ``liblatec_b200.so`` (the C ABI in ``include/latec_b200.h``).

There is no CPU fallback: importing the compute entry points on a machine
without the built library or without a CUDA device raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblatec_b200.so")

LATEC_OK = 0
ERRORS = {
    -1: (ValueError, "invalid argument"),
    -2: (RuntimeError, "CUDA error"),
    -3: (NotImplementedError, "unsupported configuration"),
    -4: (ValueError, "malformed stream"),
    -5: (RuntimeError, "workspace too small"),
    -6: (RuntimeError, "internal error"),
    -7: (ValueError, "input larger than the entry point's fixed limit"),
}
F32, F64 = 1, 2
RANS_LANES, RANS_COMPAT = 0, 1

U32, U64, I32, P, D = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_double
I64, F = ctypes.c_int64, ctypes.c_float


class QuantParams(ctypes.Structure):
    _fields_ = [("dtype", I32), ("channels", I32), ("radius", I32), ("order", I32),
                ("center", I32), ("end_mode", I32), ("round_output", I32), ("reserved", I32),
                ("round_span", D), ("round_offset", D)]


class StageStats(ctypes.Structure):
    _fields_ = [("n_out", U32), ("maxq", U32), ("done", U32), ("pad1", U32),
                ("stats", D * 5)]


class EncodeJob(ctypes.Structure):
    """latec_encode_job: one tensor of latec_encode_stages_many."""
    _fields_ = [("plan", P), ("prm", QuantParams), ("stage_eb", P), ("x", P), ("recon", P),
                ("codes", P), ("outliers", P), ("stats", P), ("hist_seg", P),
                ("hist_total", P), ("workspace", P), ("workspace_bytes", U64),
                ("max_ctas", U32), ("reserved", U32)]


class DecodeJob(ctypes.Structure):
    """latec_decode_job: one tensor of latec_decode_stages_many."""
    _fields_ = [("plan", P), ("prm", QuantParams), ("stage_eb", P), ("codes", P),
                ("outliers", P), ("out_off", P), ("n_out", P), ("recon", P), ("err", P)]


# StageStats.done bit set by a fused level encode whose plane loads did not
# arrive within the kernel's wait limit (its results are not valid).
TILE_WAIT_FAILED = 0x80000000


def check_stage_stats(stats):
    """Raise if a fused level kernel reported a failed load wait in the
    statistics of an encode (``stats``: an array of StageStats)."""
    if any(int(s.done) & TILE_WAIT_FAILED for s in stats):
        raise RuntimeError("latec_encode_stages: a fused level kernel timed out waiting for "
                           "its plane loads; the encode is invalid")


class RansStage(ctypes.Structure):
    _fields_ = [("codes_off", U64), ("out_off", U64), ("enc", U64), ("cdf", U64), ("bucket", U64),
                ("scratch_off", U64), ("blob_off", U64), ("rec_off", U64), ("framed_hi", U64),
                ("n", U32), ("K", U32), ("n_chunks", U32), ("chunk0", U32), ("alphabet", U32),
                ("kexp", I32), ("radius", I32), ("mode", I32), ("per_point", I32),
                ("blob_words", U32), ("n_out", U32), ("block0", U32)]


class Record(ctypes.Structure):
    _fields_ = [("blob", U64), ("out_at", U64), ("frame", U64), ("n", U32), ("n_out", U32),
                ("K", U32), ("n_chunks", U32), ("chunk0", U32), ("status", U32)]


class FitStage(ctypes.Structure):
    _fields_ = [("counts_off", U64), ("w_table", U64), ("seg_off", U64), ("n_segs", U32),
                ("alphabet", U32), ("kexp", I32), ("radius", I32), ("n_shapes", U32),
                ("stage", U32), ("shape_ids", U32 * 24)]


class GnnModel(ctypes.Structure):
    _fields_ = [("d", I32), ("agg_level", I32), ("params", P), ("packed_bf16", P), ("tc_err", P),
                ("packed_fp8", P), ("fp8_scales", P)]


class GnnGeom(ctypes.Structure):
    _fields_ = [("M", I32), ("L", I32), ("K", I32), ("m_tile", I32), ("n_tiles", I32),
                ("query", P), ("nbr_p", P), ("nbr_n", P), ("logd_p", P), ("logd_n", P),
                ("two", P), ("one", P), ("row_of", P), ("two_off", P), ("one_off", P),
                ("sidx_p", P), ("sidx_n", P)]


# Every symbol the header declares, with (restype, argtypes).
SIGNATURES = {
    "latec_version": (ctypes.c_char_p, []),
    "latec_launch_count": (U64, []),
    "latec_plan_create": (ctypes.c_int, [P, I32, I32, I32, I32, ctypes.POINTER(P)]),
    "latec_plan_destroy": (ctypes.c_int, [P]),
    "latec_plan_num_stages": (ctypes.c_int, [P]),
    "latec_plan_stage_info": (ctypes.c_int, [P, I32, ctypes.POINTER(U64), ctypes.POINTER(I32),
                                             ctypes.POINTER(I32), ctypes.POINTER(I32)]),
    "latec_plan_stage_flat": (ctypes.c_int, [P, I32, U64, U64, P]),
    "latec_stage_workspace_bytes": (U64, [P, I32, I32]),
    "latec_flat_workspace_bytes": (U64, [U64, I32]),
    "latec_set_row_mode": (ctypes.c_int, [I32]),
    "latec_encode_many_table_bytes": (U64, [P, I32]),
    "latec_encode_stages_many": (ctypes.c_int, [P, I32, P, U64, P]),
    "latec_decode_many_table_bytes": (U64, [P, I32]),
    "latec_decode_stages_many": (ctypes.c_int, [P, I32, P, U64, P]),
    "latec_encode_stages": (ctypes.c_int, [P, ctypes.POINTER(QuantParams), P, P, P, P, P, P, P,
                                           P, P, U64, P]),
    "latec_interp_predict_stage": (ctypes.c_int, [P, I32, ctypes.POINTER(QuantParams), P, P, P]),
    "latec_quantize": (ctypes.c_int, [ctypes.POINTER(QuantParams), D, U64, P, P, P, P, P, P, P,
                                      P, P, U64, P]),
    "latec_dequantize_workspace_bytes": (U64, [U64]),
    "latec_dequantize": (ctypes.c_int, [ctypes.POINTER(QuantParams), D, U64, P, P, P, U32, P, P,
                                        P, U64, P]),
    "latec_set_level_mode": (ctypes.c_int, [I32]),
    "latec_set_tile_mode": (ctypes.c_int, [I32]),
    "latec_set_kernel_timing": (ctypes.c_int, [I32]),
    "latec_kernel_time": (ctypes.c_int, [I32, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_uint32)]),
    "latec_decode_stages": (ctypes.c_int, [P, ctypes.POINTER(QuantParams), P, P, P, P, P, P, P,
                                           P, U64, P]),
    "latec_rans_build_tables": (ctypes.c_int, [P, I32, I32, P, P, P]),
    "latec_rans_encode_workspace_bytes": (U64, [P, I32]),
    "latec_rans_encode": (ctypes.c_int, [P, I32, P, P, P, P, I32, P, U64, P, P, P, U64, P]),
    "latec_rans_decode_workspace_bytes": (U64, [I32]),
    "latec_rans_decode": (ctypes.c_int, [P, I32, U32, P, P, P, P, P, P, U64, P]),
    "latec_fit_stage_size": (U64, []),
    "latec_fit_const": (ctypes.c_int, [P, I32, P, P, P, P, P, P, U64, P]),
    "latec_quantize_static": (ctypes.c_int, [ctypes.POINTER(QuantParams), D, U64, P, P, P, P, P,
                                             P, P, P, P]),
    "latec_scale_levels": (ctypes.c_int, [P, U64, P, I32, P, P]),
    "latec_level_order_workspace_bytes": (U64, [U64]),
    "latec_level_order": (ctypes.c_int, [P, U64, P, P, U64, P]),
    "latec_permute": (ctypes.c_int, [P, I32, P, U64, P, I32, P]),
    "latec_point_bits": (ctypes.c_int, [P, P, U64, P, U32, I32, I32, P, I32, P, P]),
    "latec_shape_costs": (ctypes.c_int, [P, P, U64, U64, P, U32, I32, I32, I32, D, P, P, I32, P,
                                         I32, P]),
    "latec_gnn_param_count": (U64, [I32, I32]),
    "latec_gnn_workspace_bytes": (U64, [I32, I32, I32, I32, I32, I32]),
    "latec_gnn_embed": (ctypes.c_int, [ctypes.POINTER(GnnModel), I32, ctypes.c_int64, P,
                                       ctypes.POINTER(GnnGeom), P, P, U64, P]),
    "latec_gnn_head": (ctypes.c_int, [ctypes.POINTER(GnnModel), I32, I32, I32, P,
                                      ctypes.c_float, P, P, P, U64, P]),
    "latec_gnn_pack_fp8": (ctypes.c_int, [P, I32, I32, I32, P, P]),
    "latec_gnn_mlp2_fp8": (ctypes.c_int, [P, I32, I64, I32, I32, P, P, P, P, P, P, P, I32, P, P]),
    "latec_gate_costs": (ctypes.c_int, [I64, P, P, P, P, P, P, D, I32, P, P, P, P]),
    "latec_gate_apply": (ctypes.c_int, [I64, P, P, P, D, I32, I32, I32, P]),
    "latec_gate_choose_apply": (ctypes.c_int, [I64, P, P, P, P, P, P, D, P, P]),
    "latec_gate_apply_word": (ctypes.c_int, [I64, P, P, P, P, P, D, P, P]),
    "latec_tr_linear": (ctypes.c_int, [P, I64, I64, I32, P, P, I32, P, I64, I32, P, P]),
    "latec_tr_linear_bwd": (ctypes.c_int, [P, I64, I64, I32, P, I32, P, I64, P, I32, P, I64, I32,
                                           P, P, P]),
    "latec_tr_linear_bf16": (ctypes.c_int, [P, I64, I64, I32, P, P, I32, P, I64, I32, P, P]),
    "latec_tr_linear_bwd_bf16": (ctypes.c_int, [P, I64, I64, I32, P, I32, P, I64, P, I32, P, I64,
                                                I32, P, P, P]),
    "latec_tr_gemm_status": (ctypes.c_int, [P]),
    "latec_tr_rows": (ctypes.c_int, [P, I64, I32, I32, I32, P, ctypes.POINTER(GnnGeom), P, I64,
                                     I32, I32, P, I32, P]),
    "latec_tr_rows_bwd": (ctypes.c_int, [P, I32, I64, I32, I32, I32, ctypes.POINTER(GnnGeom), P,
                                         I64, I32, I32, P, P, P]),
    "latec_tr_line_rows": (ctypes.c_int, [P, I32, I32, I32, I32, I64, I64, P, P]),
    "latec_tr_attn": (ctypes.c_int, [P, P, I32, P, I32, I64, F, P, P, P, P, P]),
    "latec_tr_attn_bwd": (ctypes.c_int, [P, I32, P, I32, I64, F, P, P, P, P, P, P, P, P]),
    "latec_tr_head_rows": (ctypes.c_int, [P, I64, I32, I32, P, P, P]),
    "latec_tr_head_out": (ctypes.c_int, [P, I64, I32, P, P, P, P]),
    "latec_tr_head_out_bwd": (ctypes.c_int, [P, P, I64, P, P, P, P]),
    "latec_tr_loss": (ctypes.c_int, [P, P, P, I64, I32, P, F, F, P, P, P, P]),
    "latec_tr_mix_rows": (ctypes.c_int, [P, P, I64, I32, I32, P, P]),
    "latec_tr_mix_rows_bwd": (ctypes.c_int, [P, I64, I32, I32, P, P, P]),
    "latec_tr_scatter_e": (ctypes.c_int, [P, P, I32, I32, I32, I32, I64, P, I32, P]),
    "latec_tr_adamw": (ctypes.c_int, [P, P, P, P, I64, F, F, F, F, F, I64, P]),
    "latec_tr_ema": (ctypes.c_int, [P, P, I64, F, P]),
    "latec_gnn_finalize": (ctypes.c_int, [ctypes.POINTER(GnnModel), I32, ctypes.c_int64, I32,
                                          I32, P, P, P, P, P, U64, P]),
    "latec_gnn_pack_bf16": (ctypes.c_int, [P, I32, I32, I32, P]),
    "latec_gnn_mlp2_bf16": (ctypes.c_int, [P, I32, ctypes.c_int64, I32, I32, P, P, P, P, P, I32,
                                           P, P]),
    "latec_raw_frame_bytes": (U64, [U64]),
    "latec_frame_raw": (ctypes.c_int, [P, U64, P, ctypes.c_uint32, P, U64, P]),
    "latec_unframe_raw": (ctypes.c_int, [P, U64, P, P, P]),
    "latec_record_size": (U64, []),
    "latec_parse_records": (ctypes.c_int, [P, U64, I32, I32, I32, P, P, P]),
    "latec_chunk_ranges": (ctypes.c_int, [P, P, I32, P, P, P]),
}

_lib = None


def load(require_gpu: bool = True):
    """Load the CUDA library; raise if it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C latec_b200/csrc` "
                "(the LATEC B200 codec has no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    if require_gpu:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("the LATEC B200 codec needs a CUDA device (no CPU fallback)")
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != LATEC_OK:
        exc, msg = ERRORS.get(rc, (RuntimeError, f"error {rc}"))
        raise exc(f"{what}: {msg} (code {rc})" if what else f"{msg} (code {rc})")


def ptr(t) -> int:
    """Device (or host) address of a tensor / array, 0 for None."""
    if t is None:
        return 0
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


_pinned: dict = {}


def pinned(nbytes: int, slot: str = "io"):
    """A cached page-locked host buffer of at least ``nbytes`` (per slot)."""
    import torch

    buf = _pinned.get(slot)
    if buf is None or buf.numel() < nbytes:
        size = max(int(nbytes), 1 << 20)
        size = 1 << (size - 1).bit_length()
        buf = torch.empty(size, dtype=torch.uint8, pin_memory=True)
        _pinned[slot] = buf
    return buf


def stream_ptr(stream=None) -> int:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
