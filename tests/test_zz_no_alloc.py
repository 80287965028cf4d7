"""The single-read entry point that allocates nothing (mp_realign_single_noalloc).

It is for callers that cannot allocate device memory -- a host application whose
framework already owns the GPU's memory through its own pool, or code running
where allocation is not allowed. Its scratch is a fixed array inside the library,
so these tests check, through the C ABI, that two calls in a row give the same
tuples as the regular batched entry point (mp_realign_batch) on the same reads,
within the posterior tolerance the parity tests use (1e-4), and in the same order;
that they meet the FP64 oracle's posteriors directly; and that the limits and the
too-small output lists are reported, not silently cut.
This file is collected last on purpose: a failure here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

from marginpolish_b200 import AlignmentParams, Jobs, Model, _lib, realign_batch, synth
from oracle.bindings import ExactOracle, MpoModel
from oracle.compare import check_job, check_loglik

pytestmark = pytest.mark.gpu

TOL_WEIGHT = 1e-4 * 1e7 + 1  # 1e-4 in probability, plus the floor to the integer scale


class NoallocError(Exception):
    def __init__(self, status, counts):
        super().__init__(f"status {status}")
        self.status = status
        self.counts = counts


def _noalloc_call(engine, model, params, sx, sy, anchors, strand, ragged_left=False, ragged_right=False,
                  caps=None):
    lib = _lib.load()
    sx = np.ascontiguousarray(sx, dtype=np.uint16)
    sy = np.ascontiguousarray(sy, dtype=np.uint16)
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int32).reshape(-1, 3))
    n = sx.size + sy.size
    caps = caps if caps is not None else [2 * n + 64] * 3
    bufs = [[np.zeros(max(c, 1), np.int32) for _ in range(3)] for c in caps]
    out = _lib.NoallocOutput()
    for k in range(3):
        out.weight[k] = _lib.ptr(bufs[k][0], _lib.c_int32)
        out.x[k] = _lib.ptr(bufs[k][1], _lib.c_int32)
        out.y[k] = _lib.ptr(bufs[k][2], _lib.c_int32)
        out.capacity[k] = caps[k]
    ps = params.struct()
    st = lib.mp_realign_single_noalloc(engine.handle, model.handle, ctypes.byref(ps), _lib.ptr(sx, _lib.c_uint16),
                                       sx.size, _lib.ptr(sy, _lib.c_uint16), sy.size,
                                       _lib.ptr(a, _lib.c_int32) if a.size else None, a.shape[0], int(strand),
                                       int(ragged_left), int(ragged_right), ctypes.byref(out))
    if st == _lib.MP_ERR_OVERFLOW:
        raise NoallocError(st, [int(out.count[k]) for k in range(3)])
    _lib.check(st)
    lists = [np.stack([bufs[k][0][:out.count[k]], bufs[k][1][:out.count[k]], bufs[k][2][:out.count[k]]], axis=1)
             for k in range(3)]
    return lists, out.log_likelihood, out.cells


def _same_as_batched(lists, ll, cells, ref):
    assert cells == ref.cells[0]
    assert abs(ll - ref.log_likelihood[0]) <= 1e-6 * max(1.0, abs(ref.log_likelihood[0]))
    for k in range(3):
        r = ref.job(0, k)
        assert lists[k].shape == r.shape
        assert np.array_equal(lists[k][:, 1:], r[:, 1:])  # same tuples, same order
        assert np.max(np.abs(lists[k][:, 0].astype(np.int64) - r[:, 0]), initial=0) <= TOL_WEIGHT


def test_noalloc_matches_batched_entry_point_twice(engine, polish_model):
    wl = synth.config_small(seed=7, n_reads=3)
    jobs = wl.jobs()
    model = Model.from_polish(engine, polish_model)
    params = polish_model.alignment
    eo = ExactOracle()
    mpo = (MpoModel.from_state_model(polish_model.forward), MpoModel.from_state_model(polish_model.reverse))
    for j in range(jobs.n_jobs):
        sx = jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]]
        sy = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        ref = realign_batch(engine, model, params, Jobs.single(sx, sy, a, int(jobs.strand[j])))
        oracle = eo.align_with_indels(mpo[0] if jobs.strand[j] else mpo[1], sx, sy, a, params, dense=True)
        for _call in range(2):  # two calls in a row share the library's scratch array
            lists, ll, cells = _noalloc_call(engine, model, params, sx, sy, a, jobs.strand[j])
            _same_as_batched(lists, ll, cells, ref)
            # and directly against the FP64 oracle: posteriors, completeness, reference order
            rep = check_job(lists, oracle, params.threshold)
            assert rep["max_abs_posterior_error"] <= 1e-4
            check_loglik(ll, oracle["log_likelihood"])
            assert cells == oracle["cells"]
    model.close()


def test_noalloc_ragged_ends_with_a_trimmed_rectangle(engine, default_model):
    """Ragged ends with a small split size: the rule skips the large first and last gaps, so the
    read's single rectangle is a trimmed part of the matrix ([20, 80) in both sequences here).
    The pass covers exactly that rectangle, as the batched entry point and the oracle do."""
    rng = np.random.default_rng(11)
    sx = rng.integers(0, 4, size=100).astype(np.uint16)
    sy = sx.copy()
    sub = rng.random(100) < 0.05
    sy[sub] = (sy[sub] + 1) % 4
    a = np.array([(i, i, 10) for i in range(40, 61)], dtype=np.int32)
    params = AlignmentParams(threshold=0.01, diagonal_expansion=10, split_matrix_bigger_than_this=900)
    rects = ExactOracle().split_points(a, 100, 100, 900, True, True)
    assert rects.shape[0] == 1 and tuple(rects[0]) == (20, 20, 80, 80)
    model = Model(engine, default_model, default_model)
    ref = realign_batch(engine, model, params, Jobs.single(sx, sy, a, 1, True, True))
    oracle = ExactOracle().align_with_indels(MpoModel.from_state_model(default_model), sx, sy, a, params, True, True,
                                             dense=True)
    for _call in range(2):
        lists, ll, cells = _noalloc_call(engine, model, params, sx, sy, a, 1, True, True)
        _same_as_batched(lists, ll, cells, ref)
        check_job(lists, oracle, params.threshold)
        check_loglik(ll, oracle["log_likelihood"])
        assert cells == oracle["cells"]
        assert min(int(v) for k in range(3) for v in lists[k][:, 1]) >= 19  # x - 1 of the rectangle's cells
    model.close()


def test_noalloc_reports_a_too_small_output_list(engine, polish_model):
    jobs = synth.config_small(seed=7, n_reads=1).jobs()
    model = Model.from_polish(engine, polish_model)
    params = polish_model.alignment
    sx = jobs.x_symbols[jobs.x_begin[0]:jobs.x_end[0]]
    sy = jobs.y_symbols[jobs.y_offsets[0]:jobs.y_offsets[1]]
    a = jobs.anchors[jobs.anchor_offsets[0]:jobs.anchor_offsets[1]]
    lists, _, _ = _noalloc_call(engine, model, params, sx, sy, a, jobs.strand[0])
    need = [lists[k].shape[0] for k in range(3)]
    with pytest.raises(NoallocError) as err:
        _noalloc_call(engine, model, params, sx, sy, a, jobs.strand[0], caps=[need[0] - 1, need[1], need[2]])
    assert err.value.status == _lib.MP_ERR_OVERFLOW
    assert err.value.counts == need  # the needed counts are reported
    # the array is still usable afterwards
    again, _, _ = _noalloc_call(engine, model, params, sx, sy, a, jobs.strand[0])
    for k in range(3):
        assert np.array_equal(again[k], lists[k])
    model.close()


def test_noalloc_rejects_reads_beyond_its_limit(engine, polish_model):
    model = Model.from_polish(engine, polish_model)
    sx = np.zeros(20000, np.uint16)
    sy = np.zeros(20000, np.uint16)
    with pytest.raises(_lib.MpError) as err:
        _noalloc_call(engine, model, polish_model.alignment, sx, sy, np.zeros((0, 3), np.int32), 1)
    assert err.value.status == _lib.MP_ERR_ARGUMENT
    assert "no-allocation limit" in str(err.value)
    model.close()


def test_noalloc_rejects_a_band_hull_beyond_60_slots(engine, default_model):
    """Anchors on every other diagonal cell with a fixed expansion e: the boxes between
    neighbouring anchors span x - y in [-2 - e, 2 + e], a hull of e/2 + 2 slots. e = 56 needs
    59 slots and runs; e = 58 needs 61 and is refused before any device work."""
    model = Model(engine, default_model, default_model)
    sx = np.random.default_rng(5).integers(0, 4, size=400).astype(np.uint16)
    sy = sx.copy()
    a = np.array([(i, i, 0) for i in range(0, 400, 2)], dtype=np.int32)
    ok = AlignmentParams(diagonal_expansion=56)
    _noalloc_call(engine, model, ok, sx, sy, a, 1)  # hull within the limit
    wide = AlignmentParams(diagonal_expansion=58)
    with pytest.raises(_lib.MpError) as err:
        _noalloc_call(engine, model, wide, sx, sy, a, 1)
    assert err.value.status == _lib.MP_ERR_ARGUMENT
    assert "band hull of 61 slots" in str(err.value)
    model.close()
