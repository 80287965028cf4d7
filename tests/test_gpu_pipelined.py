"""Pipelined end-to-end pass (mp_realign_batch_into): slices of the jobs alternate between two
streams; the results equal the one-shot pass's (same tuples, order, offsets, likelihoods)."""
import numpy as np
import pytest

from marginpolish_b200 import Engine, Model, realign_batch, realign_batch_pipelined, synth
from marginpolish_b200.realign import OutputBuffer

pytestmark = pytest.mark.gpu


def _check_same(a, b, n):
    for k in range(3):
        assert np.array_equal(a.offsets[k][:n + 1], b.offsets[k][:n + 1])
        assert np.array_equal(a.weight[k], b.weight[k])
        assert np.array_equal(a.x[k], b.x[k])
        assert np.array_equal(a.y[k], b.y[k])
    assert np.allclose(a.log_likelihood[:n], b.log_likelihood[:n], rtol=0, atol=0)
    assert np.array_equal(a.cells[:n], b.cells[:n])


@pytest.mark.parametrize("parts", [0, 1, 3, 7])
def test_pipelined_equals_one_shot(polish_model, parts):
    params = polish_model.alignment
    jobs = synth.config_batched(seed=13, n_chunks=5).jobs()
    eng = Engine(0)
    try:
        gm = Model.from_polish(eng, polish_model)
        want = realign_batch(eng, gm, params, jobs)
        out = OutputBuffer(pinned=True)
        for _ in range(2):  # the first call grows the buffer (capacity overflow, then again)
            got = realign_batch_pipelined(eng, gm, params, jobs, out=out, parts=parts)
            _check_same(got, want, jobs.n_jobs)
        # a different, smaller batch through the same engine and buffer
        small = synth.config_small(seed=4).jobs()
        _check_same(realign_batch_pipelined(eng, gm, params, small, out=out, parts=parts),
                    realign_batch(eng, gm, params, small), small.n_jobs)
        gm.close()
    finally:
        eng.close()


def test_pipelined_ragged_ends_and_strands(polish_model):
    """Ragged starts / ends and both strands, sliced into several parts."""
    import dataclasses
    params = polish_model.alignment
    jobs = synth.config_small(seed=9, n_reads=20).jobs()
    rng = np.random.default_rng(0)
    jobs = dataclasses.replace(jobs, ragged_left=rng.integers(0, 2, jobs.n_jobs).astype(np.uint8),
                               ragged_right=rng.integers(0, 2, jobs.n_jobs).astype(np.uint8))
    eng = Engine(0)
    try:
        gm = Model.from_polish(eng, polish_model)
        want = realign_batch(eng, gm, params, jobs)
        for parts in (2, 5):
            _check_same(realign_batch_pipelined(eng, gm, params, jobs, parts=parts), want, jobs.n_jobs)
        gm.close()
    finally:
        eng.close()
