"""Autotuner of the posterior kernel (mp_engine_autotune): per band-hull class it times the
FP32 variants (band tile shape, checkpoint stride) and warps per block on a sample batch and
makes the fastest the engine's choice. Results under the tuned choice keep the parity bar
against the FP64 oracle."""
import numpy as np
import pytest

from marginpolish_b200 import Engine, Model, realign_batch, synth
from oracle.bindings import MpoModel

from test_gpu_parity import _run_and_check

pytestmark = pytest.mark.gpu


def test_autotune_report_and_parity(polish_model):
    eng = Engine(0)
    try:
        gm = Model.from_polish(eng, polish_model)
        params = polish_model.alignment
        sample = synth.config_batched(seed=5, n_chunks=24).jobs()
        rep = eng.autotune(gm, params, sample)
        assert len(rep) >= 5
        bounds = [r["max_hull"] for r in rep]
        assert bounds == sorted(bounds) and bounds[-1] == 240
        tuned = [r for r in rep if r["candidates"] > 0]
        assert tuned, rep
        for r in tuned:
            # the class with the sample's bands was measured, and the choice holds the class
            assert r["variant"] >= 0 and r["gcups"] > 0 and r["default_gcups"] > 0
            assert r["lanes_per_task"] * r["cells_per_lane"] - 2 * r["cells_per_lane"] >= r["max_hull"]
            assert r["checkpoint_stride"] in (4, 8) and r["warps_per_block"] >= 1
            assert r["gcups"] >= 0.9 * r["default_gcups"]  # the best of the timed set (timing noise)
        # results under the tuned choice against the FP64 oracle
        jobs = synth.config_small(seed=3).jobs()
        mpo = (MpoModel.from_state_model(polish_model.forward), MpoModel.from_state_model(polish_model.reverse))
        _, worst = _run_and_check(eng, gm, mpo, jobs, params)
        assert worst <= 1e-4
        # back to the built-in choice: identical tuples to a fresh engine
        eng.autotune_reset()
        a = realign_batch(eng, gm, params, jobs)
        eng2 = Engine(0)
        try:
            gm2 = Model.from_polish(eng2, polish_model)
            b = realign_batch(eng2, gm2, params, jobs)
            for j in range(jobs.n_jobs):
                for k in range(3):
                    assert np.array_equal(a.job(j, k), b.job(j, k))
            gm2.close()
        finally:
            eng2.close()
        gm.close()
    finally:
        eng.close()
