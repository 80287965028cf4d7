"""The device-side steps of a realignment against their host forms on the same tuples.

A realignment folds every read into its chunk's graph: complete-indel candidates (poa_augment,
impl/polisher.c:354-522), matches and indels merged in read order, then the run-length estimate
(:1556-1565). With both device steps on, the candidates of all reads come from one GPU pass and
the run lengths from mp_node_update; with neither (mp_poa_set_device_steps(0)) they come from
the host threads, whose graphs the POA tests pin to the reference's. The posterior pass is
deterministic, so both forms see the same tuples and must build identical graphs.
"""
import numpy as np
import pytest

from marginpolish_b200 import Model, PoaSet, PolishParams, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gmodel(engine, polish_model):
    m = Model.from_polish(engine, polish_model)
    yield m
    m.close()


def _graph(s, c):
    return (s.nodes(c), s.observations(c), s.inserts(c), s.deletes(c), s.info(c)["score"])


def _same_graph(a, b):
    na, nb = a[0], b[0]
    assert na["bases"] == nb["bases"]
    for k in ("repeat_counts", "base_weights", "repeat_count_weights", "n_obs", "n_ins", "n_del"):
        assert np.array_equal(na[k], nb[k]), k
    assert np.array_equal(a[1], b[1])
    assert a[2] == b[2]
    assert a[3] == b[3]
    assert a[4] == b[4]


@pytest.mark.parametrize("seed,hp,rc", [(31, True, True), (32, False, False)])
def test_device_steps_build_the_host_graphs(engine, gmodel, polish_model, seed, hp, rc):
    wl = synth.config_polish(seed=seed, n_chunks=5, chunk_len=8000, coverage=30, read_len=(2000, 7000),
                             hp_runs=hp)
    pp = PolishParams(max_iterations=2, compare_repeat_counts=rc)
    sets = []
    for host in (False, True):
        s = PoaSet.from_polish_model(engine, gmodel, polish_model, pp, wl.drafts, wl.reads, wl.strands, wl.anchors)
        s.set_device_steps(run_lengths=not host, indels=not host)
        s.realign()
        sets.append(s)
    dev, hst = sets
    n_ins = 0
    for c in range(len(wl.drafts)):
        a, b = _graph(dev, c), _graph(hst, c)
        _same_graph(a, b)
        n_ins += len(a[2]) + len(a[3])
    assert n_ins > 100
    # the iterations (consensus, anchors, realignment, run lengths) stay identical
    for s in sets:
        s.iterate()
        s.estimate_repeat_counts()
    for c in range(len(wl.drafts)):
        ra, rb = dev.reference(c), hst.reference(c)
        assert ra.chars == rb.chars and np.array_equal(ra.counts, rb.counts)
        _same_graph(_graph(dev, c), _graph(hst, c))
    for s in sets:
        s.close()
