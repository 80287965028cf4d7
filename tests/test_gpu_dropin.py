"""The drop-in library called the way MarginPolish calls it: the reference's signatures,
its StateMachine (built by the reference's own code), sonLib lists of anchors in and
sonLib lists of (weight, x, y) tuples out (inc/pairwiseAligner.h:54-77, :103-106).
The host sonLib here is the project's stand-in, loaded globally as the application's.
"""
import ctypes
import os
import threading
import time
from ctypes import POINTER, Structure, c_bool, c_double, c_float, c_int, c_int64, c_uint16, c_void_p

import numpy as np
import pytest

from marginpolish_b200 import _lib, synth
from oracle.bindings import SHIM_LIB, MpoModel
from oracle.compare import check_job, check_loglik

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


class SymbolString(Structure):
    _fields_ = [("alphabet", c_void_p), ("sequence", POINTER(c_uint16)), ("length", c_int64)]


class Hmm(Structure):  # inc/stateMachine.h:138-148
    _fields_ = [("type", c_int), ("emissionsType", c_int), ("emissionNoPerState", c_void_p),
                ("emissionOffsetPerState", c_void_p), ("totalEmissions", c_int64), ("transitions", POINTER(c_double)),
                ("emissions", POINTER(c_double)), ("likelihood", c_double), ("stateNumber", c_int64)]


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
    dropin.getExpectationsUsingAnchors.argtypes = [c_void_p, POINTER(Hmm), SymbolString, SymbolString, c_void_p,
                                                   POINTER(BandingParams), c_bool, c_bool]
    dropin.getExpectations.argtypes = [c_void_p, POINTER(Hmm), SymbolString, SymbolString, POINTER(BandingParams),
                                       c_bool, c_bool]
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


def _ref_models(ref_oracle):
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    hf = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    return z, hf, hr


def test_expectations_through_the_drop_in_match_the_reference(host, ref_oracle, polish_model):
    """getExpectationsUsingAnchors / getExpectations with the reference's signature and its Hmm
    accumulator, against the reference's own getExpectationsUsingAnchors (Oracle A): the transition
    expectations within the reference's logAdd error (2e-3 relative), accumulated over reads into
    one Hmm, and the likelihood term (one total per posterior diagonal)."""
    shim, dropin = host
    z, hf, hr = _ref_models(ref_oracle)
    ap = polish_model.alignment
    bp = _params(ap)
    jobs = synth.config_small(seed=19, n_reads=3).jobs()
    trans = (c_double * 9)()
    hmm = Hmm(int(z["hmm_type"]), 0, None, None, 0, ctypes.cast(trans, POINTER(c_double)), None, 0.0, 3)
    want_t, want_ll = np.zeros(9), 0.0
    for j in range(jobs.n_jobs):
        sx = np.ascontiguousarray(jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]])
        sy = np.ascontiguousarray(jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]])
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        h = hf if jobs.strand[j] else hr
        SX = SymbolString(None, sx.ctypes.data_as(POINTER(c_uint16)), sx.size)
        SY = SymbolString(None, sy.ctypes.data_as(POINTER(c_uint16)), sy.size)
        anchors = _anchor_list(shim, a)
        dropin.getExpectationsUsingAnchors(ref_oracle.state_machine(h), ctypes.byref(hmm), SX, SY, anchors,
                                           ctypes.byref(bp), False, False)
        shim.stList_destruct(anchors)
        t, ll = ref_oracle.expectations(h, int(z["hmm_type"]), sx, sy, a, ap)
        want_t += t
        want_ll += ll
    got = np.array(trans[:])
    np.testing.assert_allclose(got, want_t, rtol=2e-3, atol=1e-6)
    assert abs(hmm.likelihood - want_ll) <= 1e-4 * abs(want_ll)
    # without anchors (getExpectations): the whole matrix of a short pair
    sx = np.ascontiguousarray(jobs.x_symbols[jobs.x_begin[0]:jobs.x_begin[0] + 60])
    sy = np.ascontiguousarray(jobs.y_symbols[jobs.y_offsets[0]:jobs.y_offsets[0] + 55])
    SX = SymbolString(None, sx.ctypes.data_as(POINTER(c_uint16)), sx.size)
    SY = SymbolString(None, sy.ctypes.data_as(POINTER(c_uint16)), sy.size)
    trans2 = (c_double * 9)()
    hmm2 = Hmm(int(z["hmm_type"]), 0, None, None, 0, ctypes.cast(trans2, POINTER(c_double)), None, 0.0, 3)
    dropin.getExpectations(ref_oracle.state_machine(hf), ctypes.byref(hmm2), SX, SY, ctypes.byref(bp), False, False)
    t, ll = ref_oracle.expectations(hf, int(z["hmm_type"]), sx, sy, np.zeros((0, 3), np.int64), ap)
    np.testing.assert_allclose(np.array(trans2[:]), t, rtol=2e-3, atol=1e-6)
    assert abs(hmm2.likelihood - ll) <= 1e-4 * abs(ll)
    ref_oracle.free_model(hf)
    ref_oracle.free_model(hr)


def test_sixteen_calling_threads_fill_the_gpu(host, ref_oracle, exact_oracle, polish_model):
    """MarginPolish calls the aligner from OpenMP threads, one chunk per thread. Driven from 16
    host threads at once, the drop-in runs at least 10x the cell rate of the same calls made one
    after another from one thread (the plain one-read-per-launch form), and the results stay
    those of the FP64 oracle."""
    shim, dropin = host
    z, hf, hr = _ref_models(ref_oracle)
    ap = polish_model.alignment
    bp = _params(ap)
    wl = synth.config_batched(seed=5, n_chunks=16, chunk_len=6000, coverage=12)
    jobs = wl.jobs()
    reads = []
    for j in range(jobs.n_jobs):
        sx = np.ascontiguousarray(jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]])
        sy = np.ascontiguousarray(jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]])
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        band = exact_oracle.band(a, sx.size, sy.size, ap.diagonal_expansion, ap.dynamic_anchor_expansion)
        cells = int(((band[:, 2] - band[:, 1]) // 2 + 1).sum())
        reads.append((sx, sy, a, bool(jobs.strand[j]), _anchor_list(shim, a), cells))
    sms = {True: ref_oracle.state_machine(hf), False: ref_oracle.state_machine(hr)}
    chunk_of = np.asarray(wl.read_template)

    def align(r, keep=None):
        sx, sy, a, fwd, anchors, _ = r
        SX = SymbolString(None, sx.ctypes.data_as(POINTER(c_uint16)), sx.size)
        SY = SymbolString(None, sy.ctypes.data_as(POINTER(c_uint16)), sy.size)
        m, gx, gy = c_void_p(), c_void_p(), c_void_p()
        dropin.getAlignedPairsWithIndelsUsingAnchors(sms[fwd], SX, SY, anchors, ctypes.byref(bp), ctypes.byref(m),
                                                     ctypes.byref(gx), ctypes.byref(gy), False, False)
        if keep is not None:
            keep.append([_read_list(shim, lst) for lst in (m, gx, gy)])
        for lst in (m, gx, gy):
            shim.stList_destruct(lst)

    # one thread, one read after another (plain form), after a warm-up call
    align(max(reads, key=lambda r: r[5]))
    plain = reads[:24]
    t = time.perf_counter()
    for r in plain:
        align(r)
    plain_rate = sum(r[5] for r in plain) / (time.perf_counter() - t)

    # 16 threads, each taking whole chunks (reads of a chunk in order), warmed up on its largest
    # read; the best of three runs, so that a moment of host-core contention on a shared machine
    # does not decide the figure
    n_threads = 16
    per_thread = [[reads[i] for i in range(len(reads)) if chunk_of[i] % n_threads == k] for k in range(n_threads)]
    barrier = threading.Barrier(n_threads + 1)
    runs = 3

    def worker(lst):
        if lst:
            align(max(lst, key=lambda r: r[5]))
        for _ in range(runs):
            barrier.wait()
            barrier.wait()
            for r in lst:
                align(r)
            barrier.wait()

    threads = [threading.Thread(target=worker, args=(lst,)) for lst in per_thread]
    for th in threads:
        th.start()
    times = []
    for _ in range(runs):
        barrier.wait()
        t = time.perf_counter()
        barrier.wait()
        barrier.wait()
        times.append(time.perf_counter() - t)
    for th in threads:
        th.join()
    multi_rate = sum(r[5] for r in reads) / min(times)
    print(f"drop-in: 1 thread {plain_rate / 1e9:.3f} GCUPS, {n_threads} threads {multi_rate / 1e9:.3f} GCUPS "
          f"({multi_rate / plain_rate:.1f}x)")
    assert multi_rate >= 10.0 * plain_rate

    # parity of the results of a threaded run on a few reads of different chunks
    sample = [reads[i] for i in np.nonzero(np.r_[True, np.diff(chunk_of) != 0])[0][:4]]
    outs = [[] for _ in sample]
    ths = [threading.Thread(target=align, args=(r, o)) for r, o in zip(sample, outs)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    for r, o in zip(sample, outs):
        sx, sy, a, fwd = r[:4]
        mpo = MpoModel.from_state_model(polish_model.forward if fwd else polish_model.reverse)
        rep = check_job(o[0], exact_oracle.align_with_indels(mpo, sx, sy, a, ap, dense=True), ap.threshold)
        assert rep["max_abs_posterior_error"] <= 1e-4
    for r in reads:
        shim.stList_destruct(r[4])
    ref_oracle.free_model(hf)
    ref_oracle.free_model(hr)
