"""The POA loop on the GPU: poa_realign / poa_realignAll in consensus mode (impl/polisher.c)
against the reference's own impl/polisher.c driving its own aligner.

* the graph built from the GPU's posterior pass carries the same nodes and nearly the same
  weights as the reference's (the reference's approximate logAdd moves posteriors by up to
  ~3e-3, so integer weights differ slightly);
* the polished consensus of every chunk is identical to the reference's;
* polishing moves an i.i.d. draft towards the truth (the reference's consensus mode, on
  homopolymer-rich drafts, mostly stops after its first iteration).
"""
import os

import numpy as np
import pytest

from marginpolish_b200 import Model, PoaSet, PolishParams, polish, synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _edit_distance(a: str, b: str) -> int:
    prev = np.arange(len(b) + 1)
    bb = np.frombuffer(b.encode(), dtype=np.uint8)
    for i, ch in enumerate(a.encode(), 1):
        cur = np.empty_like(prev)
        cur[0] = i
        sub = prev[:-1] + (bb != ch)
        cur[1:] = np.minimum(sub, prev[1:] + 1)
        # insertions along the row
        cur = np.minimum.accumulate(cur - np.arange(len(b) + 1)) + np.arange(len(b) + 1)
        prev = cur
    return int(prev[-1])


@pytest.fixture(scope="module")
def ref_poa():
    from oracle.bindings import RefPoaOracle, available_reference_poa
    if not available_reference_poa():
        pytest.skip("reference POA build (oracle/_ref/libref_poa.so) not present")
    o = RefPoaOracle()
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    o.hf = o.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    o.hr = o.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    return o


@pytest.fixture(scope="module")
def gmodel(engine, polish_model):
    m = Model.from_polish(engine, polish_model)
    yield m
    m.close()


def test_gpu_graph_close_to_reference(engine, gmodel, polish_model, ref_poa):
    ap = polish_model.alignment
    wl = synth.config_polish(seed=21, n_chunks=2, chunk_len=1200, coverage=16, read_len=(700, 1100))
    s = PoaSet.from_polish_model(engine, gmodel, polish_model, PolishParams(), wl.drafts, wl.reads, wl.strands,
                                 wl.anchors)
    s.realign()
    params_h = ref_poa.params(ref_poa.hf, ref_poa.hr, ap)
    for c in range(2):
        reads_h = ref_poa.reads(wl.reads[c], wl.strands[c])
        anchors_h = ref_poa.anchors(wl.anchors[c])
        poa = ref_poa.realign(reads_h, anchors_h, wl.drafts[c], params_h)
        a, b = s.nodes(c), ref_poa.nodes(poa)
        assert a["bases"] == b["bases"] and np.array_equal(a["repeat_counts"], b["repeat_counts"])
        # per node: |weight difference| <= 3e-3 of the integer scale per covering read
        tol = 3e-3 * 1e7 * np.maximum(1, b["n_obs"])[:, None]
        assert np.all(np.abs(a["base_weights"] - b["base_weights"]) <= tol)
        assert np.all(np.abs(a["n_obs"] - b["n_obs"]) <= 1)
        ref_poa.free_poa(poa)
        ref_poa.free_anchors(anchors_h)
        ref_poa.free_reads(reads_h)
    ref_poa.free_params(params_h)
    s.close()


@pytest.mark.parametrize("seed,hp", [(23, False), (29, True)])
def test_polished_consensus_identical_to_reference(engine, gmodel, polish_model, ref_poa, seed, hp):
    ap = polish_model.alignment
    wl = synth.config_polish(seed=seed, n_chunks=3, chunk_len=1500, coverage=20, read_len=(900, 1400), hp_runs=hp)
    pp = PolishParams(max_iterations=5)
    ours = polish(engine, gmodel, polish_model, pp, wl.drafts, wl.reads, wl.strands, wl.anchors)
    params_h = ref_poa.params(ref_poa.hf, ref_poa.hr, ap, max_iterations=5)
    improved = 0
    for c in range(3):
        reads_h = ref_poa.reads(wl.reads[c], wl.strands[c])
        anchors_h = ref_poa.anchors(wl.anchors[c])
        poa = ref_poa.realign_all(reads_h, anchors_h, wl.drafts[c], params_h)
        ref_poa.estimate_repeat_counts(poa, reads_h, params_h)
        rchars, rcounts = ref_poa.reference(poa)
        assert ours[c].chars == rchars and np.array_equal(ours[c].counts, rcounts.astype(np.uint32)), c
        truth = wl.truths[c].expand()
        improved += _edit_distance(ours[c].expand(), truth) < _edit_distance(wl.drafts[c].expand(), truth)
        ref_poa.free_poa(poa)
        ref_poa.free_anchors(anchors_h)
        ref_poa.free_reads(reads_h)
    ref_poa.free_params(params_h)
    if not hp:  # the consensus mode fixes i.i.d. drafts; on homopolymer-rich ones it rarely moves
        assert improved >= 2
