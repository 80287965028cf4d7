"""The single-read entry point that allocates nothing (mp_realign_single_noalloc).

It is for callers that cannot allocate device memory -- a host application whose
framework already owns the GPU's memory through its own pool, or code running
where allocation is not allowed. Its scratch is a fixed array inside the library,
so these tests check, through the C ABI, that two calls in a row give the same
tuples as the regular batched entry point (mp_realign_batch) on the same reads,
within the posterior tolerance the parity tests use (1e-4), and in the same order.
This file is collected last on purpose: a failure here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

from marginpolish_b200 import Jobs, Model, _lib, realign_batch, synth

pytestmark = pytest.mark.gpu

TOL_WEIGHT = 1e-4 * 1e7 + 1  # 1e-4 in probability, plus the floor to the integer scale


def _noalloc_call(engine, model, params, sx, sy, anchors, strand):
    lib = _lib.load()
    sx = np.ascontiguousarray(sx, dtype=np.uint16)
    sy = np.ascontiguousarray(sy, dtype=np.uint16)
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int32).reshape(-1, 3))
    n = sx.size + sy.size
    caps = [2 * n + 64] * 3
    bufs = [[np.zeros(c, np.int32) for _ in range(3)] for c in caps]
    out = _lib.NoallocOutput()
    for k in range(3):
        out.weight[k] = _lib.ptr(bufs[k][0], _lib.c_int32)
        out.x[k] = _lib.ptr(bufs[k][1], _lib.c_int32)
        out.y[k] = _lib.ptr(bufs[k][2], _lib.c_int32)
        out.capacity[k] = caps[k]
    ps = params.struct()
    st = lib.mp_realign_single_noalloc(engine.handle, model.handle, ctypes.byref(ps), _lib.ptr(sx, _lib.c_uint16),
                                       sx.size, _lib.ptr(sy, _lib.c_uint16), sy.size,
                                       _lib.ptr(a, _lib.c_int32) if a.size else None, a.shape[0], int(strand), 0, 0,
                                       ctypes.byref(out))
    _lib.check(st)
    lists = [np.stack([bufs[k][0][:out.count[k]], bufs[k][1][:out.count[k]], bufs[k][2][:out.count[k]]], axis=1)
             for k in range(3)]
    return lists, out.log_likelihood, out.cells


def test_noalloc_matches_batched_entry_point_twice(engine, polish_model):
    wl = synth.config_small(seed=7, n_reads=3)
    jobs = wl.jobs()
    model = Model.from_polish(engine, polish_model)
    params = polish_model.alignment
    for j in range(jobs.n_jobs):
        sx = jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]]
        sy = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        ref = realign_batch(engine, model, params, Jobs.single(sx, sy, a, int(jobs.strand[j])))
        for _call in range(2):  # two calls in a row share the library's scratch array
            lists, ll, cells = _noalloc_call(engine, model, params, sx, sy, a, jobs.strand[j])
            assert cells == ref.cells[0]
            assert abs(ll - ref.log_likelihood[0]) <= 1e-6 * max(1.0, abs(ref.log_likelihood[0]))
            for k in range(3):
                r = ref.job(0, k)
                assert lists[k].shape == r.shape
                assert np.array_equal(lists[k][:, 1:], r[:, 1:])  # same tuples, same order
                assert np.max(np.abs(lists[k][:, 0].astype(np.int64) - r[:, 0]), initial=0) <= TOL_WEIGHT
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
