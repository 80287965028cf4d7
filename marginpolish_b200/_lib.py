"""ctypes binding of the in-tree CUDA library ``libmpgpu.so`` (C ABI in include/mpgpu.h).

The library is the product; this module only declares its entry points. It is
loaded from the package directory and fails loudly when it is missing: there
is no CPU fallback for the realignment pass.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_uint8,
                    c_uint16, c_uint32, c_void_p)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpgpu.so")

MP_OK = 0
MP_ERR_ARGUMENT = 1
MP_ERR_CUDA = 2
MP_ERR_MEMORY = 3
MP_ERR_OVERFLOW = 4
MP_ERR_STATE = 5
MP_MAX_REPEAT = 51
MP_PROB_ONE = 10000000

STATUS_NAMES = {0: "MP_OK", 1: "MP_ERR_ARGUMENT", 2: "MP_ERR_CUDA", 3: "MP_ERR_MEMORY", 4: "MP_ERR_OVERFLOW",
                5: "MP_ERR_STATE"}


class MpError(RuntimeError):
    """Error status returned by the C ABI, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class ModelDesc(Structure):
    _fields_ = [
        ("log_transitions", c_double * 9),
        ("log_start", c_double * 3),
        ("log_ragged_start", c_double * 3),
        ("log_end", c_double * 3),
        ("log_ragged_end", c_double * 3),
        ("log_match", c_double * 25),
        ("log_gap_x", c_double * 5),
        ("log_gap_y", c_double * 5),
        ("run_length", c_int32),
        ("strand", c_int32),
        ("max_repeat", c_int32),
        ("reserved", c_int32),
        ("repeat_scale", c_double),
        ("repeat_log10", POINTER(c_double)),
    ]


class Params(Structure):
    _fields_ = [
        ("threshold", c_double),
        ("min_diags_between_traceback", c_int64),
        ("traceback_diagonals", c_int64),
        ("diagonal_expansion", c_int64),
        ("constraint_diagonal_trim", c_int64),
        ("split_matrix_bigger_than_this", c_int64),
        ("dynamic_anchor_expansion", c_int32),
        ("reserved", c_int32),
        ("gap_gamma", c_double),
    ]


class Batch(Structure):
    _fields_ = [
        ("n_jobs", c_int64),
        ("x_begin", POINTER(c_int64)),
        ("x_end", POINTER(c_int64)),
        ("x_symbols_length", c_int64),
        ("x_symbols", POINTER(c_uint16)),
        ("y_offsets", POINTER(c_int64)),
        ("y_symbols", POINTER(c_uint16)),
        ("anchor_offsets", POINTER(c_int64)),
        ("anchors", POINTER(c_int32)),
        ("strand", POINTER(c_uint8)),
        ("ragged_left", POINTER(c_uint8)),
        ("ragged_right", POINTER(c_uint8)),
        ("x_shift", POINTER(c_int64)),
    ]


class ResultView(Structure):
    _fields_ = [
        ("n_jobs", c_int64),
        ("offsets", POINTER(c_int64) * 3),
        ("weight", POINTER(c_int32) * 3),
        ("x", POINTER(c_int32) * 3),
        ("y", POINTER(c_int32) * 3),
        ("log_likelihood", POINTER(c_double)),
        ("cells", POINTER(c_int64)),
        ("total_cells", c_int64),
        ("device_ms", c_double),
    ]


class Output(Structure):
    _fields_ = [
        ("offsets", POINTER(c_int64) * 3),
        ("weight", POINTER(c_int32) * 3),
        ("x", POINTER(c_int32) * 3),
        ("y", POINTER(c_int32) * 3),
        ("log_likelihood", POINTER(c_double)),
        ("cells", POINTER(c_int64)),
    ]


class NoallocOutput(Structure):
    _fields_ = [
        ("weight", POINTER(c_int32) * 3),
        ("x", POINTER(c_int32) * 3),
        ("y", POINTER(c_int32) * 3),
        ("capacity", c_int64 * 3),
        ("count", c_int64 * 3),
        ("log_likelihood", c_double),
        ("cells", c_int64),
    ]


class Expectations(Structure):
    _fields_ = [
        ("transitions", (c_double * 9) * 2),
        ("match", (c_double * 25) * 2),
        ("gap_x", (c_double * 5) * 2),
        ("gap_y", (c_double * 5) * 2),
        ("start", (c_double * 3) * 2),
        ("end", (c_double * 3) * 2),
        ("repeat", (c_double * (4 * MP_MAX_REPEAT * MP_MAX_REPEAT)) * 2),
        ("log_likelihood", c_double),
    ]


class PolishParamsC(Structure):
    _fields_ = [
        ("reference_base_penalty", c_double),
        ("compare_repeat_counts", c_int32),
        ("use_run_length", c_int32),
        ("anchor_probs", POINTER(c_double)),
        ("n_anchor_probs", c_int64),
        ("min_iterations", c_int64),
        ("max_iterations", c_int64),
        ("min_polish_iterations", c_int64),
        ("max_polish_iterations", c_int64),
        ("use_read_alleles", c_int32),
        ("reserved", c_int32),
        ("candidate_variant_weight", c_double),
        ("column_anchor_trim", c_int64),
        ("filter_reads_coverage", c_int64),
        ("min_avg_base_quality", c_double),
    ]


class PolishBatch(Structure):
    _fields_ = [
        ("n_chunks", c_int64),
        ("ref_offsets", POINTER(c_int64)),
        ("ref_chars", POINTER(c_char)),
        ("ref_counts", POINTER(c_uint32)),
        ("chunk_reads", POINTER(c_int64)),
        ("read_offsets", POINTER(c_int64)),
        ("read_chars", POINTER(c_char)),
        ("read_counts", POINTER(c_uint32)),
        ("strand", POINTER(c_uint8)),
        ("anchor_offsets", POINTER(c_int64)),
        ("anchors", POINTER(c_int32)),
        ("read_qualities", POINTER(c_uint8)),
    ]


class NodeBatch(Structure):
    _fields_ = [
        ("n_chunks", c_int64),
        ("node_offsets", POINTER(c_int64)),
        ("node_bases", POINTER(c_char)),
        ("chunk_reads", POINTER(c_int64)),
        ("read_offsets", POINTER(c_int64)),
        ("read_chars", POINTER(c_char)),
        ("read_counts", POINTER(c_uint32)),
        ("strand", POINTER(c_uint8)),
        ("match_offsets", POINTER(c_int64)),
        ("weight", POINTER(c_int32)),
        ("x", POINTER(c_int32)),
        ("y", POINTER(c_int32)),
        ("max_repeat", c_int64),
        ("repeat_log10", POINTER(c_double)),
    ]


class NodeResult(Structure):
    _fields_ = [
        ("base_weights", POINTER(c_double)),
        ("repeat_weights", POINTER(c_double)),
        ("obs_offsets", POINTER(c_int64)),
        ("obs_read", POINTER(c_int64)),
        ("obs_offset", POINTER(c_int64)),
        ("obs_weight", POINTER(c_double)),
        ("repeat_counts", POINTER(ctypes.c_uint64)),
    ]


class PairBatch(Structure):
    _fields_ = [
        ("n_pairs", c_int64),
        ("x_offset", POINTER(c_int64)),
        ("x_length", POINTER(c_int32)),
        ("y_offset", POINTER(c_int64)),
        ("y_length", POINTER(c_int32)),
        ("strand", POINTER(c_uint8)),
        ("x_symbols_length", c_int64),
        ("x_symbols", POINTER(c_uint16)),
        ("y_symbols_length", c_int64),
        ("y_symbols", POINTER(c_uint16)),
    ]


class BamParamsC(Structure):
    _fields_ = [
        ("chunk_size", c_int64), ("chunk_boundary", c_int64), ("include_soft_clip", c_int32),
        ("include_secondary", c_int32), ("include_supplementary", c_int32), ("use_run_length", c_int32),
        ("min_mapq", c_int64), ("region", c_char_p),
    ]


class PoaChunkInfo(Structure):
    _fields_ = [
        ("nodes", c_int64), ("max_repeat", c_int64), ("reference_runs", c_int64), ("observations", c_int64),
        ("inserts", c_int64), ("deletes", c_int64), ("insert_runs", c_int64), ("score", c_double),
        ("iterations", c_int64),
    ]


class Tuning(Structure):
    _fields_ = [
        ("checkpoint_stride", c_int32),
        ("warps_per_block", c_int32),
        ("blocks_per_sm", c_int32),
        ("lanes_per_task", c_int32),
    ]


AUTOTUNE_MAX_CLASSES = 8


class AutotuneReport(Structure):
    _fields_ = [("n_classes", c_int32)] + [
        (name, c_int32 * AUTOTUNE_MAX_CLASSES)
        for name in ("max_hull", "tasks", "candidates", "variant", "lanes_per_task", "cells_per_lane",
                     "checkpoint_stride", "warps_per_block")
    ] + [("gcups", c_double * AUTOTUNE_MAX_CLASSES), ("default_gcups", c_double * AUTOTUNE_MAX_CLASSES)]


# Every symbol include/mpgpu.h declares (checked by the CPU tests).
EXPORTED = [
    "mp_last_error", "mp_version", "mp_engine_create", "mp_engine_destroy", "mp_engine_info",
    "mp_model_create", "mp_model_destroy", "mp_engine_set_tuning", "mp_realign_batch", "mp_result_view_get",
    "mp_result_destroy", "mp_device_batch_create", "mp_device_batch_run", "mp_device_batch_fetch",
    "mp_device_batch_stats", "mp_device_batch_destroy", "mp_band", "mp_split_points", "mp_crop_range",
    "mp_rle_encode", "mp_rle_symbols", "mp_rle_anchors", "mp_device_batch_timing", "mp_measure_fp32_peak",
    "mp_realign_single_noalloc", "mp_device_batch_reset", "mp_device_batch_counts", "mp_device_batch_fetch_into",
    "mp_host_alloc", "mp_host_free", "mp_device_batch_run_plain", "mp_forward_batch", "mp_expectations_batch",
    "mp_poa_set_create", "mp_poa_set_destroy", "mp_poa_set_realign", "mp_poa_set_realign_pairs", "mp_poa_set_iterate",
    "mp_poa_set_realign_all", "mp_poa_set_estimate_repeat_counts", "mp_poa_set_phase_seconds", "mp_poa_set_device_steps", "mp_node_update", "mp_poa_info", "mp_poa_nodes",
    "mp_poa_observations", "mp_poa_inserts", "mp_poa_deletes", "mp_poa_reference", "mp_poa_consensus",
    "mp_poa_anchor_alignments", "mp_engine_autotune", "mp_engine_autotune_reset",
    "mp_engine_set_graph_capture", "mp_realign_batch_into", "mp_engine_release_buffers", "mp_forward_pairs",
    "mp_forward_pairs_timing", "mp_measure_fp64_peak", "mp_poa_set_iterate_polish", "mp_poa_set_build_bubbles", "mp_poa_set_score_bubbles", "mp_poa_bubble_sizes",
    "mp_poa_bubbles", "mp_poa_bubble_consensus", "mp_merge_contig", "mp_match_pairs_reference",
    "mp_bam_open", "mp_bam_close", "mp_bam_chunk_count", "mp_bam_chunk", "mp_bam_convert", "mp_bam_reads_sizes",
    "mp_bam_reads",
]

_lib = None


def load() -> ctypes.CDLL:
    """Loads libmpgpu.so from the package directory (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with marginpolish_b200.build.build() "
                          "(nvcc, sm_100a); there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    P = POINTER
    sig = {
        "mp_last_error": (c_char_p, []),
        "mp_version": (c_char_p, []),
        "mp_engine_create": (c_int, [c_int, P(c_void_p)]),
        "mp_engine_destroy": (None, [c_void_p]),
        "mp_engine_info": (c_int, [c_void_p, P(c_int), P(c_int), P(c_int)]),
        "mp_engine_release_buffers": (c_int, [c_void_p]),
        "mp_engine_set_tuning": (c_int, [c_void_p, P(Tuning)]),
        "mp_engine_autotune": (c_int, [c_void_p, c_void_p, P(Params), P(Batch), P(AutotuneReport)]),
        "mp_engine_autotune_reset": (c_int, [c_void_p]),
        "mp_engine_set_graph_capture": (c_int, [c_void_p, c_int]),
        "mp_model_create": (c_int, [c_void_p, P(ModelDesc), P(ModelDesc), P(c_void_p)]),
        "mp_model_destroy": (None, [c_void_p]),
        "mp_realign_batch": (c_int, [c_void_p, c_void_p, P(Params), P(Batch), P(c_void_p)]),
        "mp_result_view_get": (c_int, [c_void_p, P(ResultView)]),
        "mp_result_destroy": (None, [c_void_p]),
        "mp_device_batch_create": (c_int, [c_void_p, c_void_p, P(Params), P(Batch), P(c_void_p)]),
        "mp_device_batch_run": (c_int, [c_void_p, c_void_p, P(c_float)]),
        "mp_device_batch_fetch": (c_int, [c_void_p, c_void_p, P(c_void_p)]),
        "mp_device_batch_stats": (c_int, [c_void_p, P(c_int64), P(c_int64), P(c_int32)]),
        "mp_device_batch_destroy": (None, [c_void_p]),
        "mp_device_batch_reset": (c_int, [c_void_p, c_void_p, P(Params), P(Batch)]),
        "mp_device_batch_counts": (c_int, [c_void_p, P(c_int64)]),
        "mp_device_batch_fetch_into": (c_int, [c_void_p, c_void_p, P(Output)]),
        "mp_realign_batch_into": (c_int, [c_void_p, c_void_p, P(Params), P(Batch), ctypes.c_int32, P(Output),
                                          P(c_int64), P(c_int64)]),
        "mp_host_alloc": (c_int, [ctypes.c_size_t, P(c_void_p)]),
        "mp_host_free": (None, [c_void_p]),
        "mp_device_batch_run_plain": (c_int, [c_void_p, c_void_p, c_int64, P(c_float), P(c_int64)]),
        "mp_device_batch_timing": (c_int, [c_void_p, P(c_float), P(c_float)]),
        "mp_measure_fp32_peak": (c_int, [c_void_p, P(c_double)]),
        "mp_measure_fp64_peak": (c_int, [c_void_p, P(c_double)]),
        "mp_realign_single_noalloc": (c_int, [c_void_p, c_void_p, P(Params), P(c_uint16), c_int64, P(c_uint16),
                                              c_int64, P(c_int32), c_int64, c_int, c_int, c_int, P(NoallocOutput)]),
        "mp_forward_batch": (c_int, [c_void_p, c_void_p, P(Params), P(Batch), P(c_double)]),
        "mp_expectations_batch": (c_int, [c_void_p, c_void_p, P(Params), P(Batch), P(Expectations), P(c_double)]),
        "mp_poa_set_create": (c_int, [c_void_p, c_void_p, P(Params), P(PolishParamsC), P(PolishBatch), P(c_double),
                                      P(c_void_p)]),
        "mp_poa_set_destroy": (None, [c_void_p]),
        "mp_poa_set_realign": (c_int, [c_void_p]),
        "mp_poa_set_realign_pairs": (c_int, [c_void_p, P(P(c_int64)), P(P(c_int64))]),
        "mp_poa_set_iterate": (c_int, [c_void_p]),
        "mp_poa_set_iterate_polish": (c_int, [c_void_p]),
        "mp_poa_set_build_bubbles": (c_int, [c_void_p]),
        "mp_poa_set_score_bubbles": (c_int, [c_void_p]),
        "mp_poa_bubble_sizes": (c_int, [c_void_p, c_int64, P(c_int64)]),
        "mp_poa_bubbles": (c_int, [c_void_p, c_int64, P(c_int64), P(c_int64), P(c_char), P(ctypes.c_uint64),
                                   P(c_int64), P(c_double), P(c_float)]),
        "mp_poa_bubble_consensus": (c_int, [c_void_p, c_int64, P(c_int64), P(c_char), P(ctypes.c_uint64), c_int64,
                                            P(c_int64), P(c_int64)]),
        "mp_forward_pairs": (c_int, [c_void_p, c_void_p, P(PairBatch), P(c_double)]),
        "mp_match_pairs_reference": (c_int, [c_void_p, c_void_p, P(Params), P(Batch), P(c_int64), P(c_int32),
                                             P(c_int32), P(c_int32), c_int64, P(c_int64)]),
        "mp_merge_contig": (c_int, [c_void_p, c_void_p, P(Params), c_int64, P(c_int64), c_char_p, c_int64, c_int64,
                                    P(c_char), c_int64, P(c_int64), P(c_int64)]),
        "mp_forward_pairs_timing": (c_int, [c_void_p, P(c_float), P(c_int64), P(c_int64)]),
        "mp_bam_open": (c_int, [c_char_p, P(BamParamsC), P(c_void_p)]),
        "mp_bam_close": (None, [c_void_p]),
        "mp_bam_chunk_count": (c_int, [c_void_p, P(c_int64)]),
        "mp_bam_chunk": (c_int, [c_void_p, c_int64, P(c_char), c_int64, P(c_int64)]),
        "mp_bam_convert": (c_int, [c_void_p, c_int64, c_int64, P(c_int64), c_char_p, c_int64, ctypes.c_uint64]),
        "mp_bam_reads_sizes": (c_int, [c_void_p, c_int64, P(c_int64)]),
        "mp_bam_reads": (c_int, [c_void_p, c_int64, P(c_int64), P(c_char), P(c_uint32), P(c_uint8), P(c_uint8),
                                 P(c_uint8), P(c_int64), P(c_int32), P(c_int64), P(c_char)]),
        "mp_poa_set_realign_all": (c_int, [c_void_p]),
        "mp_poa_set_estimate_repeat_counts": (c_int, [c_void_p]),
        "mp_poa_set_phase_seconds": (c_int, [c_void_p, P(c_double), c_int64]),
        "mp_poa_set_device_steps": (c_int, [c_void_p, c_int32]),
        "mp_node_update": (c_int, [c_void_p, P(NodeBatch), P(NodeResult)]),
        "mp_poa_info": (c_int, [c_void_p, c_int64, P(PoaChunkInfo)]),
        "mp_poa_nodes": (c_int, [c_void_p, c_int64, P(c_char), P(ctypes.c_uint64), P(c_double), P(c_double),
                                 P(c_int64), P(c_int64), P(c_int64)]),
        "mp_poa_observations": (c_int, [c_void_p, c_int64, P(c_int64), P(c_int64), P(c_double)]),
        "mp_poa_inserts": (c_int, [c_void_p, c_int64, P(c_double), P(c_double), P(c_int64), P(c_char),
                                   P(ctypes.c_uint64), P(c_int64)]),
        "mp_poa_deletes": (c_int, [c_void_p, c_int64, P(c_int64), P(c_double), P(c_double), P(c_int64)]),
        "mp_poa_reference": (c_int, [c_void_p, c_int64, P(c_char), P(ctypes.c_uint64)]),
        "mp_poa_consensus": (c_int, [c_void_p, c_int64, P(c_char), P(ctypes.c_uint64), c_int64, P(c_int64),
                                     P(c_int64)]),
        "mp_poa_anchor_alignments": (c_int, [c_void_p, c_int64, P(c_int64), P(c_int64), P(c_int64), c_int64,
                                             P(c_int64)]),
        "mp_band": (c_int, [P(c_int32), c_int64, c_int64, c_int64, c_int64, c_int, P(c_int64)]),
        "mp_split_points": (c_int, [P(c_int32), c_int64, c_int64, c_int64, c_int64, c_int, c_int, P(c_int64),
                                    c_int64, P(c_int64)]),
        "mp_crop_range": (c_int, [P(c_int32), c_int64, c_int64, c_int64, P(c_int64), P(c_int64)]),
        "mp_rle_encode": (c_int, [c_char_p, c_int64, P(c_char), P(c_uint32), P(c_int64)]),
        "mp_rle_symbols": (c_int, [P(c_char), P(c_uint32), c_int64, c_int, c_uint32, P(c_uint16)]),
        "mp_rle_anchors": (c_int, [P(c_int64), c_int64, P(c_uint32), c_int64, P(c_uint32), c_int64, P(c_int32),
                                   P(c_int64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    """Raises MpError with the library's message for a non-OK status."""
    if status != MP_OK:
        msg = load().mp_last_error()
        raise MpError(status, msg.decode() if msg else "")


def ptr(arr, ctype):
    """ctypes pointer to a contiguous numpy array (None -> NULL)."""
    if arr is None:
        return None
    return arr.ctypes.data_as(POINTER(ctype))
