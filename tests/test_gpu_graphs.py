"""CUDA graph capture of the device-resident pass (mp_engine_set_graph_capture): replayed runs
and runs after a reset to a different batch give the same tuples as direct launches."""
import numpy as np
import pytest

from marginpolish_b200 import DeviceBatch, Engine, Model, synth

pytestmark = pytest.mark.gpu


def _pairs(db):
    r = db.fetch()
    return [(r.weight[k].copy(), r.x[k].copy(), r.y[k].copy(), r.offsets[k].copy()) for k in range(3)]


def _same(a, b):
    return all(all(np.array_equal(u, v) for u, v in zip(a[k], b[k])) for k in range(3))


def test_graph_replay_and_update_match_direct_launches(polish_model):
    params = polish_model.alignment
    first = synth.config_batched(seed=11, n_chunks=6).jobs()
    second = synth.config_small(seed=2).jobs()
    direct = Engine(0)
    graphs = Engine(0)
    graphs.set_graph_capture(True)
    try:
        md, mg = Model.from_polish(direct, polish_model), Model.from_polish(graphs, polish_model)
        dd = DeviceBatch(direct, md, params, first)
        dg = DeviceBatch(graphs, mg, params, first)
        dd.run()
        want = _pairs(dd)
        for _ in range(3):  # capture, then replays
            assert dg.run() > 0.0
            assert _same(_pairs(dg), want)
        # a different batch: the graph is captured again (updated in place when the shape allows)
        dd.reset(second)
        dg.reset(second)
        dd.run()
        dg.run()
        assert _same(_pairs(dg), _pairs(dd))
        dg.run()
        assert _same(_pairs(dg), _pairs(dd))
        for x in (dd, dg, md, mg):
            x.close()
    finally:
        direct.close()
        graphs.close()
