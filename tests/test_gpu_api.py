"""The batch API around the posterior kernel: reusable device batches (reset), result
counts, fetching into caller-owned (page-locked or pageable) host arrays, and the one-shot
calls that reuse the engine's cached batch. Every path must give the same tuples as a
fresh batch fetched through the C ABI's result object."""
import ctypes

import numpy as np
import pytest

from marginpolish_b200 import DeviceBatch, Model, _lib, realign_batch, synth
from marginpolish_b200.realign import OutputBuffer, _copy_view

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.total_cells == b.total_cells
    assert np.array_equal(a.cells, b.cells)
    assert np.allclose(a.log_likelihood, b.log_likelihood, rtol=0, atol=0)
    for k in range(3):
        assert np.array_equal(a.offsets[k], b.offsets[k])
        assert np.array_equal(a.weight[k], b.weight[k])
        assert np.array_equal(a.x[k], b.x[k])
        assert np.array_equal(a.y[k], b.y[k])


def _fresh(engine, model, params, jobs):
    db = DeviceBatch(engine, model, params, jobs)
    db.run()
    r = db.fetch()
    db.close()
    return r


def test_reset_counts_and_fetch_into(engine, polish_model):
    model = Model.from_polish(engine, polish_model)
    params = polish_model.alignment
    big = synth.config_small(seed=5, n_reads=8).jobs()
    small = synth.config_small(seed=6, n_reads=3).jobs()
    ref_big, ref_small = _fresh(engine, model, params, big), _fresh(engine, model, params, small)

    db = DeviceBatch(engine, model, params, big)
    db.run()
    totals = db.counts()
    assert totals == [int(ref_big.offsets[k][-1]) for k in range(3)]
    pinned = OutputBuffer(pinned=True)
    _same(db.fetch_into(pinned), ref_big)
    _same(db.fetch_into(OutputBuffer(pinned=False)), ref_big)
    # a smaller batch in the same device buffers, then the larger one again
    db.reset(small)
    db.run()
    _same(db.fetch_into(pinned), ref_small)
    db.reset(big)
    db.run()
    _same(db.fetch_into(pinned), ref_big)
    db.close()
    model.close()


def test_one_shot_calls_reuse_the_engine_batch(engine, polish_model):
    model = Model.from_polish(engine, polish_model)
    params = polish_model.alignment
    a = synth.config_small(seed=8, n_reads=4).jobs()
    b = synth.config_small(seed=9, n_reads=6).jobs()
    ref_a, ref_b = _fresh(engine, model, params, a), _fresh(engine, model, params, b)
    out = OutputBuffer(pinned=True)
    _same(realign_batch(engine, model, params, a, out=out), ref_a)
    _same(realign_batch(engine, model, params, b), ref_b)
    _same(realign_batch(engine, model, params, a), ref_a)
    # the C ABI's one-shot call (result object owned by the library)
    lib = _lib.load()
    ps, bs, res = params.struct(), b.struct(), ctypes.c_void_p()
    _lib.check(lib.mp_realign_batch(engine.handle, model.handle, ctypes.byref(ps), ctypes.byref(bs),
                                    ctypes.byref(res)))
    try:
        _same(_copy_view(lib, res), ref_b)
    finally:
        lib.mp_result_destroy(res)
    model.close()


def test_fetch_before_run_is_a_state_error(engine, polish_model):
    model = Model.from_polish(engine, polish_model)
    db = DeviceBatch(engine, model, polish_model.alignment, synth.config_small(seed=10, n_reads=2).jobs())
    with pytest.raises(_lib.MpError) as err:
        db.counts()
    assert err.value.status == _lib.MP_ERR_STATE
    db.close()
    model.close()


def test_argument_errors_are_reported(engine, polish_model):
    """Malformed jobs come back as MP_ERR_ARGUMENT with a message: anchors not strictly
    increasing, an anchor outside the matrix, an odd expansion under dynamic anchor expansion
    (all found by the planner), and a repeat count at the run-length table's limit (found by
    the kernel, which clamps the lookup and flags the task)."""
    from marginpolish_b200 import Jobs
    model = Model.from_polish(engine, polish_model)
    params = polish_model.alignment
    sx = np.array([(1 << 8) | b for b in (0, 1, 2, 3, 0, 1, 2, 3)], np.uint16)
    sy = sx.copy()
    cases = {
        "not strictly increasing": np.array([[2, 2, 4], [2, 3, 4]], np.int32),
        "outside the matrix": np.array([[2, 2, 4], [8, 7, 4]], np.int32),
        "odd expansion": np.array([[2, 2, 3]], np.int32),
    }
    for what, anchors in cases.items():
        jobs = Jobs.single(sx, sy, anchors)
        with pytest.raises(_lib.MpError) as err:
            realign_batch(engine, model, params, jobs)
        assert err.value.status == _lib.MP_ERR_ARGUMENT, what
    big = sx.copy()
    big[3] = (51 << 8) | 3  # observed repeat count 51: beyond the 51 x 51 table
    with pytest.raises(_lib.MpError) as err:
        realign_batch(engine, model, params, Jobs.single(big, sy, np.zeros((0, 3), np.int32)))
    assert err.value.status == _lib.MP_ERR_ARGUMENT
    # the engine still works after the errors
    ok = realign_batch(engine, model, params, Jobs.single(sx, sy, np.array([[2, 2, 4]], np.int32)))
    assert ok.total_cells > 0
    model.close()
