"""ctypes bindings of the two CPU oracles -- TEST INFRASTRUCTURE ONLY.

Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() import
this module, and only as the checker of the CUDA library.

* ``RefOracle``  (Oracle A): the reference's own impl/pairwiseAligner.c and
  impl/stateMachine.c compiled unmodified (oracle/_ref/libref_oracle.so).
* ``ExactOracle`` (Oracle B): the FP64 restatement in oracle/phmm_oracle.c
  (oracle/libmp_oracle.so); with the reference's logAdd plugged in it must
  reproduce Oracle A bit for bit.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_double, c_int, c_int64, c_uint8, c_uint16, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref_oracle.so")
REF_LIB_CHECKED = os.path.join(HERE, "_ref", "libref_oracle_checked.so")
EXACT_LIB = os.path.join(HERE, "libmp_oracle.so")
SHIM_LIB = os.path.join(HERE, "libsonlib_shim.so")


def _p(a, t):
    return a.ctypes.data_as(POINTER(t)) if a is not None else None


class OracleParams(Structure):
    """Layout shared by RefoParams (ref_harness.c) and MpoParams (phmm_oracle.h)."""

    _fields_ = [
        ("threshold", c_double),
        ("minDiagsBetweenTraceBack", c_int64),
        ("traceBackDiagonals", c_int64),
        ("diagonalExpansion", c_int64),
        ("constraintDiagonalTrim", c_int64),
        ("splitMatrixBiggerThanThis", c_int64),
        ("dynamicAnchorExpansion", c_int64),
        ("gapGamma", c_double),
    ]

    @classmethod
    def from_alignment(cls, ap) -> "OracleParams":
        return cls(ap.threshold, ap.min_diags_between_traceback, ap.traceback_diagonals, ap.diagonal_expansion,
                   ap.constraint_diagonal_trim, ap.split_matrix_bigger_than_this,
                   1 if ap.dynamic_anchor_expansion else 0, ap.gap_gamma)


class _Pairs(Structure):
    _fields_ = [("n", c_int64 * 3), ("t", POINTER(c_int64) * 3)]


class _MpoResult(Structure):
    _fields_ = [("n", c_int64 * 3), ("t", POINTER(c_int64) * 3), ("logLikelihood", c_double), ("cells", c_int64),
                ("nDense", c_int64), ("dense", POINTER(c_double))]


class MpoModel(Structure):
    _fields_ = [
        ("trans", c_double * 9), ("start", c_double * 3), ("raggedStart", c_double * 3), ("end", c_double * 3),
        ("raggedEnd", c_double * 3), ("match", c_double * 25), ("gapX", c_double * 5), ("gapY", c_double * 5),
        ("runLength", c_int64), ("strand", c_int64), ("maxRepeat", c_int64), ("repeatScale", c_double),
        ("repeat10", POINTER(c_double)),
    ]

    @classmethod
    def from_state_model(cls, sm) -> "MpoModel":
        m = cls()
        m.trans[:] = list(map(float, sm.log_transitions))
        m.start[:] = list(map(float, sm.log_start))
        m.raggedStart[:] = list(map(float, sm.log_ragged_start))
        m.end[:] = list(map(float, sm.log_end))
        m.raggedEnd[:] = list(map(float, sm.log_ragged_end))
        m.match[:] = list(map(float, sm.log_match))
        m.gapX[:] = list(map(float, sm.log_gap_x))
        m.gapY[:] = list(map(float, sm.log_gap_y))
        m.runLength = 1 if sm.run_length else 0
        m.strand = int(sm.strand)
        m.maxRepeat = 51
        m.repeatScale = float(sm.repeat_scale)
        if sm.run_length:
            tab = np.ascontiguousarray(sm.repeat_log10, dtype=np.float64).reshape(-1)
            m._keep = tab
            m.repeat10 = _p(tab, c_double)
        return m


def _tuples(ptr, n):
    if n == 0:
        return np.zeros((0, 3), dtype=np.int64)
    return np.ctypeslib.as_array(ptr, shape=(n * 3,)).reshape(n, 3).copy()


def available_reference() -> bool:
    return os.path.exists(REF_LIB)


class RefOracle:
    """Oracle A: the reference's own code."""

    def __init__(self, checked: bool = False):
        path = REF_LIB_CHECKED if checked else REF_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build with `make -C oracle reference`")
        lib = ctypes.CDLL(path)
        P = POINTER
        lib.refo_model_create.restype = c_void_p
        lib.refo_model_create.argtypes = [c_int, P(c_double), P(c_double), c_int, P(c_double), c_int]
        lib.refo_model_create_default.restype = c_void_p
        lib.refo_model_destroy.argtypes = [c_void_p]
        for f in ("refo_model_match_emission",):
            getattr(lib, f).restype = c_double
            getattr(lib, f).argtypes = [c_void_p, c_int, c_int]
        for f in ("refo_model_gap_x_emission", "refo_model_gap_y_emission"):
            getattr(lib, f).restype = c_double
            getattr(lib, f).argtypes = [c_void_p, c_int]
        lib.refo_model_boundary.restype = c_double
        lib.refo_model_boundary.argtypes = [c_void_p, c_int, c_int]
        lib.refo_model_transitions.argtypes = [c_void_p, P(c_double)]
        job = [c_void_p, P(c_uint16), c_int64, P(c_uint16), c_int64, P(c_int64), c_int64, P(OracleParams), c_int, c_int]
        for f in ("refo_align_with_indels", "refo_align"):
            getattr(lib, f).restype = P(_Pairs)
            getattr(lib, f).argtypes = job
        lib.refo_pairs_free.argtypes = [P(_Pairs)]
        lib.refo_align_batch.restype = c_int64
        lib.refo_align_batch.argtypes = [c_void_p, c_void_p, c_int64, P(c_int64), P(c_uint16), P(c_int64),
                                         P(c_uint16), P(c_int64), P(c_int64), P(c_uint8), P(OracleParams), c_int,
                                         P(c_int64), c_void_p]
        lib.refo_align_chunks.restype = c_int64
        lib.refo_align_chunks.argtypes = [c_void_p, c_void_p, c_int64, P(c_int64), P(c_int64), P(c_uint16),
                                          P(c_int64), P(c_uint16), P(c_int64), P(c_int64), P(c_uint8),
                                          P(OracleParams), c_int, P(c_int64)]
        lib.refo_band.argtypes = [P(c_int64), c_int64, c_int64, c_int64, c_int64, c_int, P(c_int64)]
        lib.refo_split_points.restype = c_int64
        lib.refo_split_points.argtypes = [P(c_int64), c_int64, c_int64, c_int64, c_int64, c_int, c_int, P(c_int64),
                                          c_int64]
        lib.refo_logadd.restype = c_double
        lib.refo_logadd.argtypes = [c_double, c_double]
        lib.refo_forward_probability.restype = c_double
        lib.refo_forward_probability.argtypes = job
        lib.refo_expectations.argtypes = [c_void_p, c_int, P(c_uint16), c_int64, P(c_uint16), c_int64, P(c_int64),
                                          c_int64, P(OracleParams), c_int, c_int, P(c_double), P(c_double)]
        lib.refo_mea.restype = c_int64
        lib.refo_mea.argtypes = [P(c_int64), c_int64, P(c_int64), c_int64, P(c_int64), c_int64, c_int64, c_int64,
                                 c_double, P(c_double), P(c_int64), c_int64]
        self.lib = lib

    # ---- models ----
    def model(self, hmm_type, transitions, emissions, reverse_complement, repeat_log10=None, strand=1):
        t = np.ascontiguousarray(transitions, dtype=np.float64)
        e = np.ascontiguousarray(emissions, dtype=np.float64)
        r = None if repeat_log10 is None else np.ascontiguousarray(repeat_log10, dtype=np.float64).reshape(-1)
        h = self.lib.refo_model_create(hmm_type, _p(t, c_double), _p(e, c_double), 1 if reverse_complement else 0,
                                       _p(r, c_double), 1 if strand else 0)
        return h

    def default_model(self):
        return self.lib.refo_model_create_default()

    def free_model(self, h):
        self.lib.refo_model_destroy(h)

    def transitions(self, h) -> np.ndarray:
        out = np.zeros(9)
        self.lib.refo_model_transitions(h, _p(out, c_double))
        return out

    def match_emission(self, h, cx, cy):
        return self.lib.refo_model_match_emission(h, cx, cy)

    def gap_emissions(self, h, c):
        return self.lib.refo_model_gap_x_emission(h, c), self.lib.refo_model_gap_y_emission(h, c)

    def boundary(self, h, which):
        return np.array([self.lib.refo_model_boundary(h, which, s) for s in range(3)])

    # ---- alignment ----
    def align_with_indels(self, h, sx, sy, anchors, params, ragged_left=False, ragged_right=False):
        sx = np.ascontiguousarray(sx, dtype=np.uint16)
        sy = np.ascontiguousarray(sy, dtype=np.uint16)
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        op = OracleParams.from_alignment(params)
        r = self.lib.refo_align_with_indels(h, _p(sx, c_uint16), sx.size, _p(sy, c_uint16), sy.size,
                                            _p(a, c_int64), a.shape[0], ctypes.byref(op), int(ragged_left),
                                            int(ragged_right))
        out = tuple(_tuples(r.contents.t[k], r.contents.n[k]) for k in range(3))
        self.lib.refo_pairs_free(r)
        return out

    def align_batch(self, hf, hr, jobs, params, n_threads=0):
        """OpenMP over jobs; returns per-job tuple counts (n, 3)."""
        n = jobs.n_jobs
        xoff_b = np.ascontiguousarray(jobs.x_begin, dtype=np.int64)
        # the harness takes x offsets as (begin, next); build contiguous copies per job
        xs, xo = _gather_x(jobs)
        op = OracleParams.from_alignment(params)
        counts = np.zeros((n, 3), dtype=np.int64)
        an = np.ascontiguousarray(jobs.anchors, dtype=np.int64)
        self.lib.refo_align_batch(hf, hr, n, _p(xo, c_int64), _p(xs, c_uint16), _p(jobs.y_offsets, c_int64),
                                  _p(jobs.y_symbols, c_uint16), _p(jobs.anchor_offsets, c_int64), _p(an, c_int64),
                                  _p(jobs.strand, c_uint8), ctypes.byref(op), n_threads, _p(counts, c_int64), None)
        del xoff_b
        return counts

    def align_chunks(self, hf, hr, jobs, chunk_offsets, params, n_threads=0):
        """OpenMP over chunks (schedule(dynamic,1)), the reads of a chunk in order on one thread,
        as marginPolish.c:436-439 runs poa_realign; chunk c is jobs chunk_offsets[c] ..
        chunk_offsets[c+1]-1. Returns per-job tuple counts (n, 3)."""
        n = jobs.n_jobs
        xs, xo = _gather_x(jobs)
        op = OracleParams.from_alignment(params)
        counts = np.zeros((n, 3), dtype=np.int64)
        an = np.ascontiguousarray(jobs.anchors, dtype=np.int64)
        co = np.ascontiguousarray(chunk_offsets, dtype=np.int64)
        assert co[0] == 0 and co[-1] == n
        self.lib.refo_align_chunks(hf, hr, co.size - 1, _p(co, c_int64), _p(xo, c_int64), _p(xs, c_uint16),
                                   _p(jobs.y_offsets, c_int64), _p(jobs.y_symbols, c_uint16),
                                   _p(jobs.anchor_offsets, c_int64), _p(an, c_int64), _p(jobs.strand, c_uint8),
                                   ctypes.byref(op), n_threads, _p(counts, c_int64))
        return counts

    def band(self, anchors, lx, ly, expansion, dynamic):
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        out = np.zeros((lx + ly + 1, 3), dtype=np.int64)
        self.lib.refo_band(_p(a, c_int64), a.shape[0], lx, ly, expansion, int(dynamic), _p(out, c_int64))
        return out

    def band_cells(self, anchors, lx, ly, expansion, dynamic) -> int:
        """Cells of one job's band from the reference's own band construction: the sum over
        anti-diagonals of (xmyR - xmyL) / 2 + 1."""
        if lx + ly == 0:
            return 0
        b = self.band(anchors, lx, ly, expansion, dynamic)
        return int(((b[:, 2] - b[:, 1]) // 2 + 1).sum())

    def split_points(self, anchors, lx, ly, max_size, ragged_left, ragged_right):
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        n = self.lib.refo_split_points(_p(a, c_int64), a.shape[0], lx, ly, max_size, int(ragged_left),
                                       int(ragged_right), None, 0)
        out = np.zeros((max(n, 1), 4), dtype=np.int64)
        self.lib.refo_split_points(_p(a, c_int64), a.shape[0], lx, ly, max_size, int(ragged_left),
                                   int(ragged_right), _p(out, c_int64), n)
        return out[:n]

    def logadd_address(self) -> int:
        return ctypes.cast(self.lib.refo_logadd, c_void_p).value

    def state_machine(self, h) -> int:
        """Address of the reference StateMachine of a model handle (for the drop-in tests)."""
        self.lib.refo_model_state_machine.restype = c_void_p
        self.lib.refo_model_state_machine.argtypes = [c_void_p]
        return self.lib.refo_model_state_machine(h)

    def forward_probability(self, h, sx, sy, anchors, params, ragged_left=False, ragged_right=False) -> float:
        """The reference's computeForwardProbability (impl/pairwiseAligner.c:813-865)."""
        sx = np.ascontiguousarray(sx, dtype=np.uint16)
        sy = np.ascontiguousarray(sy, dtype=np.uint16)
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        op = OracleParams.from_alignment(params)
        return self.lib.refo_forward_probability(h, _p(sx, c_uint16), sx.size, _p(sy, c_uint16), sy.size,
                                                 _p(a, c_int64), a.shape[0], ctypes.byref(op), int(ragged_left),
                                                 int(ragged_right))

    def expectations(self, h, hmm_type, sx, sy, anchors, params, ragged_left=False, ragged_right=False):
        """The reference's getExpectationsUsingAnchors: (9 transition counts, its likelihood sum)."""
        sx = np.ascontiguousarray(sx, dtype=np.uint16)
        sy = np.ascontiguousarray(sy, dtype=np.uint16)
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        op = OracleParams.from_alignment(params)
        t = np.zeros(9)
        lk = c_double(0.0)
        self.lib.refo_expectations(h, hmm_type, _p(sx, c_uint16), sx.size, _p(sy, c_uint16), sy.size,
                                   _p(a, c_int64), a.shape[0], ctypes.byref(op), int(ragged_left), int(ragged_right),
                                   _p(t, c_double), ctypes.byref(lk))
        return t, lk.value


def _gather_x(jobs):
    """Per-job contiguous X symbols and monotone offsets (the oracle harness layout)."""
    parts = [jobs.x_symbols[b:e] for b, e in zip(jobs.x_begin, jobs.x_end)]
    xo = np.zeros(len(parts) + 1, dtype=np.int64)
    xo[1:] = np.cumsum([p.size for p in parts])
    xs = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(1, np.uint16), dtype=np.uint16)
    return xs, xo


class ExactOracle:
    """Oracle B: FP64 restatement (exact log-sum unless a logAdd function pointer is given)."""

    def __init__(self):
        if not os.path.exists(EXACT_LIB):
            raise FileNotFoundError(f"{EXACT_LIB} missing: build with `make -C oracle oracle-b`")
        lib = ctypes.CDLL(EXACT_LIB)
        P = POINTER
        lib.mpo_align_with_indels.restype = P(_MpoResult)
        lib.mpo_align_with_indels.argtypes = [P(MpoModel), P(c_uint16), c_int64, P(c_uint16), c_int64, P(c_int64),
                                              c_int64, P(OracleParams), c_int, c_int, c_void_p, c_int]
        lib.mpo_result_free.argtypes = [P(_MpoResult)]
        lib.mpo_band.restype = c_int
        lib.mpo_band.argtypes = [P(c_int64), c_int64, c_int64, c_int64, c_int64, c_int, P(c_int64)]
        lib.mpo_split_points.restype = c_int64
        lib.mpo_split_points.argtypes = [P(c_int64), c_int64, c_int64, c_int64, c_int64, c_int, c_int, P(c_int64),
                                         c_int64]
        lib.mpo_match_emission.restype = c_double
        lib.mpo_match_emission.argtypes = [P(MpoModel), c_uint16, c_uint16]
        lib.mpo_gap_x_emission.restype = c_double
        lib.mpo_gap_x_emission.argtypes = [P(MpoModel), c_uint16]
        lib.mpo_gap_y_emission.restype = c_double
        lib.mpo_gap_y_emission.argtypes = [P(MpoModel), c_uint16]
        lib.mpo_forward_probability.restype = c_double
        lib.mpo_forward_probability.argtypes = [P(MpoModel), P(c_uint16), c_int64, P(c_uint16), c_int64, P(c_int64),
                                                c_int64, c_int64, c_int, c_int, c_int, c_void_p]
        lib.mpo_expectations.restype = c_double
        lib.mpo_expectations.argtypes = [P(MpoModel), P(c_uint16), c_int64, P(c_uint16), c_int64, P(c_int64),
                                         c_int64, c_int64, c_int, c_int, c_int, P(c_double)]
        lib.mpo_align_batch.restype = c_int64
        lib.mpo_align_batch.argtypes = [P(MpoModel), P(MpoModel), c_int64, P(c_int64), P(c_uint16), P(c_int64),
                                        P(c_uint16), P(c_int64), P(c_int64), P(c_uint8), P(OracleParams), c_int,
                                        P(c_int64), P(c_double)]
        self.lib = lib

    def align_with_indels(self, model: MpoModel, sx, sy, anchors, params, ragged_left=False, ragged_right=False,
                          logadd=None, dense=False):
        sx = np.ascontiguousarray(sx, dtype=np.uint16)
        sy = np.ascontiguousarray(sy, dtype=np.uint16)
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        op = OracleParams.from_alignment(params)
        r = self.lib.mpo_align_with_indels(ctypes.byref(model), _p(sx, c_uint16), sx.size, _p(sy, c_uint16), sy.size,
                                           _p(a, c_int64), a.shape[0], ctypes.byref(op), int(ragged_left),
                                           int(ragged_right), logadd, 2 if dense == "near" else (1 if dense else 0))
        rc = r.contents
        out = {
            "pairs": tuple(_tuples(rc.t[k], rc.n[k]) for k in range(3)),
            "log_likelihood": rc.logLikelihood,
            "cells": rc.cells,
        }
        if dense:
            out["dense"] = (np.ctypeslib.as_array(rc.dense, shape=(rc.nDense * 5,)).reshape(-1, 5).copy()
                            if rc.nDense else np.zeros((0, 5)))
        self.lib.mpo_result_free(r)
        return out

    def align_batch(self, mf: MpoModel, mr: MpoModel, jobs, params, n_threads=0):
        n = jobs.n_jobs
        xs, xo = _gather_x(jobs)
        op = OracleParams.from_alignment(params)
        counts = np.zeros((n, 3), dtype=np.int64)
        ll = np.zeros(n)
        an = np.ascontiguousarray(jobs.anchors, dtype=np.int64)
        self.lib.mpo_align_batch(ctypes.byref(mf), ctypes.byref(mr), n, _p(xo, c_int64), _p(xs, c_uint16),
                                 _p(jobs.y_offsets, c_int64), _p(jobs.y_symbols, c_uint16),
                                 _p(jobs.anchor_offsets, c_int64), _p(an, c_int64), _p(jobs.strand, c_uint8),
                                 ctypes.byref(op), n_threads, _p(counts, c_int64), _p(ll, c_double))
        return counts, ll

    def band(self, anchors, lx, ly, expansion, dynamic):
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        out = np.zeros((lx + ly + 1, 3), dtype=np.int64)
        rc = self.lib.mpo_band(_p(a, c_int64), a.shape[0], lx, ly, expansion, int(dynamic), _p(out, c_int64))
        return out if rc == 0 else None

    def split_points(self, anchors, lx, ly, max_size, ragged_left, ragged_right):
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        n = self.lib.mpo_split_points(_p(a, c_int64), a.shape[0], lx, ly, max_size, int(ragged_left),
                                      int(ragged_right), None, 0)
        out = np.zeros((max(n, 1), 4), dtype=np.int64)
        self.lib.mpo_split_points(_p(a, c_int64), a.shape[0], lx, ly, max_size, int(ragged_left),
                                  int(ragged_right), _p(out, c_int64), n)
        return out[:n]

    def forward_probability(self, model: MpoModel, sx, sy, anchors, expansion, dynamic=False, ragged_left=False,
                            ragged_right=False, logadd=None) -> float:
        """ln P over the band (band_construct when not dynamic), FP64, exact log-sum unless logadd."""
        sx = np.ascontiguousarray(sx, dtype=np.uint16)
        sy = np.ascontiguousarray(sy, dtype=np.uint16)
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        return self.lib.mpo_forward_probability(ctypes.byref(model), _p(sx, c_uint16), sx.size, _p(sy, c_uint16),
                                                sy.size, _p(a, c_int64), a.shape[0], int(expansion), int(dynamic),
                                                int(ragged_left), int(ragged_right), logadd)

    def expectations(self, model: MpoModel, sx, sy, anchors, expansion, dynamic=True, ragged_left=False,
                     ragged_right=False):
        """Exact FP64 expected counts over the whole band: (ln P, dict of count arrays)."""
        sx = np.ascontiguousarray(sx, dtype=np.uint16)
        sy = np.ascontiguousarray(sy, dtype=np.uint16)
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        out = np.zeros(50 + 4 * 51 * 51)
        lp = self.lib.mpo_expectations(ctypes.byref(model), _p(sx, c_uint16), sx.size, _p(sy, c_uint16), sy.size,
                                       _p(a, c_int64), a.shape[0], int(expansion), int(dynamic), int(ragged_left),
                                       int(ragged_right), _p(out, c_double))
        return lp, {"transitions": out[0:9].copy(), "match": out[9:34].copy(), "gap_x": out[34:39].copy(),
                    "gap_y": out[39:44].copy(), "start": out[44:47].copy(), "end": out[47:50].copy(),
                    "repeat": out[50:].copy()}


REF_POA_LIB = os.path.join(HERE, "_ref", "libref_poa.so")


def available_reference_poa() -> bool:
    return os.path.exists(REF_POA_LIB)


class RefPoaOracle:
    """The reference's own POA steps (impl/polisher.c and impl/bubbleGraph.c compiled unmodified,
    oracle/_ref/libref_poa.so): poa_realign, poa_getConsensus, poa_getAnchorAlignments, the
    run-length estimate, the bubble graph of poa_polish and poa_realignAll in consensus and
    polish mode."""

    def __init__(self):
        if not os.path.exists(REF_POA_LIB):
            raise FileNotFoundError(f"{REF_POA_LIB} missing: build with `make -C oracle reference`")
        lib = ctypes.CDLL(REF_POA_LIB)
        P = POINTER
        from ctypes import c_char, c_char_p, c_uint32, c_uint64
        self._c_char, self._c_uint64 = c_char, c_uint64
        lib.refo_model_create.restype = c_void_p
        lib.refo_model_create.argtypes = [c_int, P(c_double), P(c_double), c_int, P(c_double), c_int]
        lib.refo_model_destroy.argtypes = [c_void_p]
        lib.refo_align_with_indels.restype = P(_Pairs)
        lib.refo_align_with_indels.argtypes = [c_void_p, P(c_uint16), c_int64, P(c_uint16), c_int64, P(c_int64),
                                               c_int64, P(OracleParams), c_int, c_int]
        lib.refo_pairs_free.argtypes = [P(_Pairs)]
        lib.refpoa_params_create.restype = c_void_p
        lib.refpoa_params_create.argtypes = [c_void_p, c_void_p, P(OracleParams), c_int, c_double, c_int, P(c_double),
                                             c_int64, c_int64, c_int64]
        lib.refpoa_params_destroy.argtypes = [c_void_p]
        lib.refpoa_reads_create.restype = c_void_p
        lib.refpoa_reads_create.argtypes = [c_int64, c_char_p, P(c_uint32), P(c_int64), P(c_uint8)]
        lib.refpoa_reads_destroy.argtypes = [c_void_p]
        lib.refpoa_anchors_create.restype = c_void_p
        lib.refpoa_anchors_create.argtypes = [c_int64, P(c_int64), P(c_int64)]
        lib.refpoa_anchors_destroy.argtypes = [c_void_p]
        for f in ("refpoa_realign", "refpoa_realign_all"):
            getattr(lib, f).restype = c_void_p
            getattr(lib, f).argtypes = [c_void_p, c_void_p, c_char_p, P(c_uint32), c_int64, c_void_p]
        lib.refpoa_destroy.argtypes = [c_void_p]
        lib.refpoa_estimate_repeat_counts.argtypes = [c_void_p, c_void_p, c_void_p]
        lib.refpoa_score.restype = c_double
        lib.refpoa_score.argtypes = [c_void_p]
        lib.refpoa_reference.restype = c_int64
        lib.refpoa_reference.argtypes = [c_void_p, P(c_char), P(c_uint64), c_int64]
        lib.refpoa_node_count.restype = c_int64
        lib.refpoa_node_count.argtypes = [c_void_p]
        lib.refpoa_max_repeat.restype = c_int64
        lib.refpoa_max_repeat.argtypes = [c_void_p]
        lib.refpoa_nodes.argtypes = [c_void_p, P(c_char), P(c_uint64), P(c_double), P(c_double), P(c_int64),
                                     P(c_int64), P(c_int64)]
        lib.refpoa_observations.argtypes = [c_void_p, P(c_int64), P(c_int64), P(c_double)]
        lib.refpoa_inserts.restype = c_int64
        lib.refpoa_inserts.argtypes = [c_void_p, P(c_double), P(c_double), P(c_int64), P(c_char), P(c_uint64),
                                       P(c_int64)]
        lib.refpoa_deletes.argtypes = [c_void_p, P(c_int64), P(c_double), P(c_double), P(c_int64)]
        lib.refpoa_consensus.restype = c_int64
        lib.refpoa_consensus.argtypes = [c_void_p, c_void_p, P(c_char), P(c_uint64), c_int64, P(c_int64)]
        lib.refpoa_anchor_alignments.restype = c_int64
        lib.refpoa_anchor_alignments.argtypes = [c_void_p, P(c_int64), c_int64, c_void_p, P(c_int64), P(c_int64),
                                                 c_int64]
        lib.refpoa_params_set_polish.argtypes = [c_void_p, c_int, c_double, c_int64, c_int64, c_double, c_int64,
                                                 c_int64, c_int64]
        lib.refpoa_reads_set_qualities.argtypes = [c_void_p, P(c_uint8), P(c_int64)]
        lib.refpoa_bubble_graph.restype = c_void_p
        lib.refpoa_bubble_graph.argtypes = [c_void_p, c_void_p, c_void_p]
        lib.refpoa_bubble_graph_destroy.argtypes = [c_void_p]
        lib.refpoa_bubble_count.restype = c_int64
        lib.refpoa_bubble_count.argtypes = [c_void_p]
        lib.refpoa_bubble_info.argtypes = [c_void_p, c_int64] + [P(c_int64)] * 4
        lib.refpoa_bubble_allele.restype = c_int64
        lib.refpoa_bubble_allele.argtypes = [c_void_p, c_int64, c_int64, P(c_char), P(c_uint64), c_int64]
        lib.refpoa_bubble_reads.argtypes = [c_void_p, c_int64, c_void_p, P(c_int64), P(c_int64), P(c_int64),
                                            P(c_double)]
        lib.refpoa_bubble_supports.argtypes = [c_void_p, c_int64, P(ctypes.c_float)]
        lib.refpoa_remove_overlap.restype = c_int64
        lib.refpoa_remove_overlap.argtypes = [c_char_p, c_char_p, c_int64, c_void_p, P(c_int64), P(c_int64)]
        lib.refpoa_bubble_consensus.restype = c_int64
        lib.refpoa_bubble_consensus.argtypes = [c_void_p, c_void_p, P(c_uint64), P(c_char), P(c_uint64), c_int64,
                                                P(c_int64)]
        self.lib = lib

    # ---- construction ----
    def model(self, hmm_type, transitions, emissions, reverse_complement, repeat_log10=None, strand=1):
        t = np.ascontiguousarray(transitions, dtype=np.float64)
        e = np.ascontiguousarray(emissions, dtype=np.float64)
        r = None if repeat_log10 is None else np.ascontiguousarray(repeat_log10, dtype=np.float64).reshape(-1)
        return self.lib.refo_model_create(hmm_type, _p(t, c_double), _p(e, c_double), 1 if reverse_complement else 0,
                                          _p(r, c_double), 1 if strand else 0)

    def free_model(self, h):
        self.lib.refo_model_destroy(h)

    def params(self, hf, hr, alignment, use_rle=True, penalty=0.5, compare_repeat_counts=True,
               anchor_probs=(0.9, 10, 0.95, 4, 0.99, 0), min_iterations=0, max_iterations=5):
        op = OracleParams.from_alignment(alignment)
        pr = np.ascontiguousarray(anchor_probs, dtype=np.float64)
        return self.lib.refpoa_params_create(hf, hr, ctypes.byref(op), int(use_rle), float(penalty),
                                             int(compare_repeat_counts), _p(pr, c_double), pr.size, int(min_iterations),
                                             int(max_iterations))

    def free_params(self, h):
        self.lib.refpoa_params_destroy(h)

    def set_polish(self, params_h, polish):
        """The polish-mode fields of the parameters from a PolishParams (use_read_alleles,
        candidate_variant_weight, column_anchor_trim, filter_reads_coverage,
        min_avg_base_quality, max_consensus_strings, min/max_polish_iterations)."""
        self.lib.refpoa_params_set_polish(params_h, int(polish.use_read_alleles), float(polish.candidate_variant_weight),
                                          int(polish.column_anchor_trim), int(polish.filter_reads_coverage),
                                          float(polish.min_avg_base_quality), int(polish.max_consensus_strings),
                                          int(polish.min_polish_iterations), int(polish.max_polish_iterations))

    def set_qualities(self, reads_h, qualities):
        """Per-run qualities of every read (a list of uint8 arrays, one per read run)."""
        off = np.zeros(len(qualities) + 1, np.int64)
        off[1:] = np.cumsum([len(q) for q in qualities])
        flat = np.ascontiguousarray(np.concatenate([np.asarray(q, np.uint8) for q in qualities])
                                    if off[-1] else np.zeros(1, np.uint8))
        self.lib.refpoa_reads_set_qualities(reads_h, _p(flat, c_uint8), _p(off, c_int64))

    def bubble_graph(self, poa, reads_h, params_h):
        """bubbleGraph_constructFromPoa, exported: a list of bubbles, each a dict with ref_start,
        ref_length, alleles (list of (chars, counts)), reads (rows read, start, length), quals
        and supports (alleles x reads, float32); plus the consensus path, the new consensus and
        the POA-to-consensus map of bubbleGraph_getConsensusPath / getConsensusString."""
        from ctypes import c_float
        bg = self.lib.refpoa_bubble_graph(poa, reads_h, params_h)
        out = []
        for i in range(self.lib.refpoa_bubble_count(bg)):
            v = [c_int64() for _ in range(4)]
            self.lib.refpoa_bubble_info(bg, i, *[ctypes.byref(x) for x in v])
            ref_start, ref_len, n_al, n_rd = (x.value for x in v)
            alleles = []
            for j in range(n_al):
                n = self.lib.refpoa_bubble_allele(bg, i, j, None, None, 0)
                chars = (self._c_char * max(n, 1))()
                counts = np.zeros(max(n, 1), np.uint64)
                self.lib.refpoa_bubble_allele(bg, i, j, chars, _p(counts, self._c_uint64), n)
                alleles.append((bytes(chars[:n]), counts[:n].copy()))
            rd = np.zeros((3, max(n_rd, 1)), np.int64)
            q = np.zeros(max(n_rd, 1), np.float64)
            self.lib.refpoa_bubble_reads(bg, i, reads_h, _p(rd[0], c_int64), _p(rd[1], c_int64), _p(rd[2], c_int64),
                                         _p(q, c_double))
            sup = np.zeros(max(n_al * n_rd, 1), np.float32)
            self.lib.refpoa_bubble_supports(bg, i, _p(sup, c_float))
            out.append(dict(ref_start=ref_start, ref_length=ref_len, alleles=alleles,
                            reads=rd[:, :n_rd].T.copy(), quals=q[:n_rd].copy(),
                            supports=sup[:n_al * n_rd].reshape(n_al, n_rd).copy()))
        n_nodes = self.lib.refpoa_node_count(poa)
        path = np.zeros(max(len(out), 1), np.uint64)
        cap = 4 * n_nodes + 64
        chars = (self._c_char * cap)()
        counts = np.zeros(cap, np.uint64)
        node_map = np.zeros(max(n_nodes - 1, 1), np.int64)
        n = self.lib.refpoa_bubble_consensus(bg, params_h, _p(path, self._c_uint64), chars,
                                             _p(counts, self._c_uint64), cap, _p(node_map, c_int64))
        assert n <= cap
        self.lib.refpoa_bubble_graph_destroy(bg)
        return dict(bubbles=out, path=path[:len(out)].astype(np.int64), chars=bytes(chars[:n]),
                    counts=counts[:n].copy(), map=node_map[:n_nodes - 1].copy())

    def remove_overlap(self, prefix: str, suffix: str, overlap: int, params_h):
        """removeOverlap: (overlap match weight, prefix crop end, suffix crop start)."""
        a, b = c_int64(0), c_int64(0)
        w = self.lib.refpoa_remove_overlap(prefix.encode(), suffix.encode(), int(overlap), params_h, ctypes.byref(a),
                                           ctypes.byref(b))
        return int(w), a.value, b.value

    def reads(self, rle_reads, strands):
        from ctypes import c_uint32
        off = np.zeros(len(rle_reads) + 1, np.int64)
        off[1:] = np.cumsum([len(r) for r in rle_reads])
        chars = b"".join(r.chars for r in rle_reads) or b"\0"
        counts = np.ascontiguousarray(np.concatenate([np.asarray(r.counts, np.uint32) for r in rle_reads])
                                      if rle_reads else np.zeros(1, np.uint32), dtype=np.uint32)
        st = np.ascontiguousarray(strands, dtype=np.uint8)
        return self.lib.refpoa_reads_create(len(rle_reads), chars, _p(counts, c_uint32), _p(off, c_int64),
                                            _p(st, c_uint8))

    def free_reads(self, h):
        self.lib.refpoa_reads_destroy(h)

    def anchors(self, per_read):
        lists = [np.asarray(a, dtype=np.int64).reshape(-1, 3) for a in per_read]
        off = np.zeros(len(lists) + 1, np.int64)
        off[1:] = np.cumsum([a.shape[0] for a in lists])
        flat = np.ascontiguousarray(np.concatenate(lists) if lists and off[-1] else np.zeros((1, 3), np.int64))
        return self.lib.refpoa_anchors_create(len(lists), _p(off, c_int64), _p(flat, c_int64))

    def free_anchors(self, h):
        self.lib.refpoa_anchors_destroy(h)

    def align_with_indels(self, h, sx, sy, anchors, params):
        """The reference aligner of this library (the one poa_realign calls)."""
        sx = np.ascontiguousarray(sx, dtype=np.uint16)
        sy = np.ascontiguousarray(sy, dtype=np.uint16)
        a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int64).reshape(-1, 3))
        op = OracleParams.from_alignment(params)
        r = self.lib.refo_align_with_indels(h, _p(sx, c_uint16), sx.size, _p(sy, c_uint16), sy.size, _p(a, c_int64),
                                            a.shape[0], ctypes.byref(op), 0, 0)
        out = tuple(_tuples(r.contents.t[k], r.contents.n[k]) for k in range(3))
        self.lib.refo_pairs_free(r)
        return out

    # ---- the loop ----
    def realign(self, reads_h, anchors_h, ref, params_h):
        from ctypes import c_uint32
        c = np.ascontiguousarray(ref.counts, dtype=np.uint32) if len(ref) else np.zeros(1, np.uint32)
        return self.lib.refpoa_realign(reads_h, anchors_h, ref.chars or b"\0", _p(c, c_uint32), len(ref), params_h)

    def realign_all(self, reads_h, anchors_h, ref, params_h):
        """poa_realignAll; anchors_h None aligns every read to the whole reference (no anchors)."""
        from ctypes import c_uint32
        c = np.ascontiguousarray(ref.counts, dtype=np.uint32) if len(ref) else np.zeros(1, np.uint32)
        return self.lib.refpoa_realign_all(reads_h, anchors_h, ref.chars or b"\0", _p(c, c_uint32), len(ref),
                                           params_h)

    def free_poa(self, h):
        self.lib.refpoa_destroy(h)

    def estimate_repeat_counts(self, poa, reads_h, params_h):
        self.lib.refpoa_estimate_repeat_counts(poa, reads_h, params_h)

    def score(self, poa):
        return self.lib.refpoa_score(poa)

    def reference(self, poa):
        n = self.lib.refpoa_reference(poa, None, None, 0)
        chars = (self._c_char * max(n, 1))()
        counts = np.zeros(max(n, 1), np.uint64)
        self.lib.refpoa_reference(poa, chars, _p(counts, self._c_uint64), n)
        return bytes(chars[:n]), counts[:n].copy()

    def nodes(self, poa):
        n = self.lib.refpoa_node_count(poa)
        m = self.lib.refpoa_max_repeat(poa)
        bases = (self._c_char * max(n, 1))()
        rc = np.zeros(n, np.uint64)
        bw = np.zeros((n, 5))
        rcw = np.zeros((n, m))
        no, ni, nd = (np.zeros(n, np.int64) for _ in range(3))
        self.lib.refpoa_nodes(poa, bases, _p(rc, self._c_uint64), _p(bw, c_double), _p(rcw, c_double),
                              _p(no, c_int64), _p(ni, c_int64), _p(nd, c_int64))
        return {"bases": bytes(bases[:n]), "repeat_counts": rc, "base_weights": bw, "repeat_count_weights": rcw,
                "n_obs": no, "n_ins": ni, "n_del": nd}

    def observations(self, poa):
        k = int(self.nodes(poa)["n_obs"].sum())
        r, o, w = np.zeros(k, np.int64), np.zeros(k, np.int64), np.zeros(k)
        self.lib.refpoa_observations(poa, _p(r, c_int64), _p(o, c_int64), _p(w, c_double))
        return np.stack([r, o, w], axis=1) if k else np.zeros((0, 3))

    def inserts(self, poa):
        k = int(self.nodes(poa)["n_ins"].sum())
        runs = self.lib.refpoa_inserts(poa, None, None, None, None, None, None)
        wf, wr = np.zeros(max(k, 1)), np.zeros(max(k, 1))
        ln, no = np.zeros(max(k, 1), np.int64), np.zeros(max(k, 1), np.int64)
        chars = (self._c_char * max(runs, 1))()
        counts = np.zeros(max(runs, 1), np.uint64)
        self.lib.refpoa_inserts(poa, _p(wf, c_double), _p(wr, c_double), _p(ln, c_int64), chars,
                                _p(counts, self._c_uint64), _p(no, c_int64))
        out, at = [], 0
        raw = bytes(chars[:runs])
        for i in range(k):
            out.append((raw[at:at + ln[i]], tuple(int(v) for v in counts[at:at + ln[i]]), float(wf[i]), float(wr[i]),
                        int(no[i])))
            at += int(ln[i])
        return out

    def deletes(self, poa):
        k = int(self.nodes(poa)["n_del"].sum())
        ln, no = np.zeros(max(k, 1), np.int64), np.zeros(max(k, 1), np.int64)
        wf, wr = np.zeros(max(k, 1)), np.zeros(max(k, 1))
        self.lib.refpoa_deletes(poa, _p(ln, c_int64), _p(wf, c_double), _p(wr, c_double), _p(no, c_int64))
        return [(int(ln[i]), float(wf[i]), float(wr[i]), int(no[i])) for i in range(k)]

    def consensus(self, poa, params_h):
        n = self.lib.refpoa_node_count(poa)
        cap = 64 * n + 64
        chars = (self._c_char * cap)()
        counts = np.zeros(cap, np.uint64)
        m = np.zeros(max(n - 1, 1), np.int64)
        k = self.lib.refpoa_consensus(poa, params_h, chars, _p(counts, self._c_uint64), cap, _p(m, c_int64))
        return bytes(chars[:k]), counts[:k].copy(), m[:n - 1].copy()

    def anchor_alignments(self, poa, node_map, n_reads, params_h):
        mp = None if node_map is None else np.ascontiguousarray(node_map, dtype=np.int64)
        cap = int(self.nodes(poa)["n_obs"].sum()) + 1
        off = np.zeros(n_reads + 1, np.int64)
        tri = np.zeros((cap, 3), np.int64)
        self.lib.refpoa_anchor_alignments(poa, _p(mp, c_int64), n_reads, params_h, _p(off, c_int64), _p(tri, c_int64),
                                          cap)
        return [tri[off[r]:off[r + 1]].copy() for r in range(n_reads)]
