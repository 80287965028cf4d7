"""The drop-in library called the way MarginPolish calls it: the reference's signatures,
its StateMachine (built by the reference's own code), sonLib lists of anchors in and
sonLib lists of (weight, x, y) tuples out (inc/pairwiseAligner.h:54-77, :103-106).
The host sonLib here is the project's stand-in, loaded globally as the application's.
"""
import ctypes
import os
from ctypes import POINTER, Structure, c_bool, c_double, c_float, c_int64, c_uint16, c_void_p

import numpy as np
import pytest

from marginpolish_b200 import _lib, synth
from oracle.bindings import SHIM_LIB, MpoModel
from oracle.compare import check_job, check_loglik

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


class SymbolString(Structure):
    _fields_ = [("alphabet", c_void_p), ("sequence", POINTER(c_uint16)), ("length", c_int64)]


class BandingParams(Structure):  # PairwiseAlignmentParameters (inc/pairwiseAligner.h:28-39)
    _fields_ = [("threshold", c_double), ("minDiagsBetweenTraceBack", c_int64), ("traceBackDiagonals", c_int64),
                ("diagonalExpansion", c_int64), ("constraintDiagonalTrim", c_int64),
                ("splitMatrixBiggerThanThis", c_int64), ("alignAmbiguityCharacters", c_bool), ("gapGamma", c_float),
                ("dynamicAnchorExpansion", c_bool)]


@pytest.fixture(scope="module")
def host():
    shim = ctypes.CDLL(SHIM_LIB, mode=ctypes.RTLD_GLOBAL)
    shim.stList_construct3.restype = c_void_p
    shim.stList_construct3.argtypes = [c_int64, c_void_p]
    shim.stList_append.argtypes = [c_void_p, c_void_p]
    shim.stList_length.restype = c_int64
    shim.stList_length.argtypes = [c_void_p]
    shim.stList_get.restype = c_void_p
    shim.stList_get.argtypes = [c_void_p, c_int64]
    shim.stList_destruct.argtypes = [c_void_p]
    shim.stIntTuple_construct3.restype = c_void_p
    shim.stIntTuple_construct3.argtypes = [c_int64, c_int64, c_int64]
    shim.stIntTuple_get.restype = c_int64
    shim.stIntTuple_get.argtypes = [c_void_p, c_int64]
    dropin = ctypes.CDLL(os.path.join(os.path.dirname(_lib.LIB_PATH), "libmpgpu_dropin.so"))
    dropin.getAlignedPairsWithIndelsUsingAnchors.argtypes = [c_void_p, SymbolString, SymbolString, c_void_p,
                                                             POINTER(BandingParams), POINTER(c_void_p),
                                                             POINTER(c_void_p), POINTER(c_void_p), c_bool, c_bool]
    dropin.computeForwardProbability.restype = c_double
    dropin.computeForwardProbability.argtypes = [SymbolString, SymbolString, c_void_p, POINTER(BandingParams),
                                                 c_void_p, c_bool, c_bool]
    return shim, dropin


def _anchor_list(shim, a):
    lst = shim.stList_construct3(0, None)
    for x, y, e in np.asarray(a, dtype=np.int64).reshape(-1, 3):
        shim.stList_append(lst, shim.stIntTuple_construct3(int(x), int(y), int(e)))
    return lst


def _read_list(shim, lst):
    n = shim.stList_length(lst)
    out = np.zeros((n, 3), dtype=np.int64)
    for i in range(n):
        t = shim.stList_get(lst, i)
        out[i] = [shim.stIntTuple_get(t, k) for k in range(3)]
    return out


def _params(ap):
    return BandingParams(ap.threshold, ap.min_diags_between_traceback, ap.traceback_diagonals, ap.diagonal_expansion,
                         ap.constraint_diagonal_trim, ap.split_matrix_bigger_than_this, False, ap.gap_gamma,
                         bool(ap.dynamic_anchor_expansion))


def test_reference_signatures_through_the_drop_in(host, ref_oracle, exact_oracle, polish_model):
    shim, dropin = host
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    hf = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    ap = polish_model.alignment
    bp = _params(ap)
    jobs = synth.config_small(seed=43, n_reads=4).jobs()
    for j in range(jobs.n_jobs):
        sx = np.ascontiguousarray(jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]])
        sy = np.ascontiguousarray(jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]])
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        fwd = bool(jobs.strand[j])
        sm = ref_oracle.state_machine(hf if fwd else hr)
        SX = SymbolString(None, sx.ctypes.data_as(POINTER(c_uint16)), sx.size)
        SY = SymbolString(None, sy.ctypes.data_as(POINTER(c_uint16)), sy.size)
        anchors = _anchor_list(shim, a)
        m, gx, gy = c_void_p(), c_void_p(), c_void_p()
        dropin.getAlignedPairsWithIndelsUsingAnchors(sm, SX, SY, anchors, ctypes.byref(bp), ctypes.byref(m),
                                                     ctypes.byref(gx), ctypes.byref(gy), False, False)
        got = [_read_list(shim, lst) for lst in (m, gx, gy)]
        mpo = MpoModel.from_state_model(polish_model.forward if fwd else polish_model.reverse)
        o = exact_oracle.align_with_indels(mpo, sx, sy, a, ap, dense=True)
        rep = check_job(got, o, ap.threshold)
        assert rep["max_abs_posterior_error"] <= 1e-4
        lp = dropin.computeForwardProbability(SX, SY, anchors, ctypes.byref(bp), sm, False, False)
        check_loglik(lp, exact_oracle.forward_probability(mpo, sx, sy, a, ap.diagonal_expansion, False))
        for lst in (m, gx, gy, anchors):
            shim.stList_destruct(lst)
    ref_oracle.free_model(hf)
    ref_oracle.free_model(hr)
