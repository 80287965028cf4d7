"""Device-side node update (mp_node_update) against the reference's poa_augment and run-length
estimate, and against this library's host graph on large random batches.

The match part of poa_augment (impl/polisher.c:322-340) gives each node its base and run-length
weights and its observation list; poa_estimateRepeatCountsUsingBayesianModel (:1556-1565,
:1796-1865) picks every node's run length from its observations. The GPU version must give the
same doubles, the same observation order and the same run lengths, bit for bit.
"""
import os

import numpy as np
import pytest

from marginpolish_b200 import PoaSet, PolishParams, synth
from marginpolish_b200._lib import MpError
from marginpolish_b200.poa import node_update
from marginpolish_b200.rle import RleString, crop_range

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def ref_poa():
    from oracle.bindings import RefPoaOracle, available_reference_poa
    if not available_reference_poa():
        pytest.skip("reference POA build (oracle/_ref/libref_poa.so) not present")
    return RefPoaOracle()


@pytest.fixture(scope="module")
def ref_models(ref_poa):
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    hf = ref_poa.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref_poa.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    yield hf, hr
    ref_poa.free_model(hf)
    ref_poa.free_model(hr)


def _reference_matches(ref_poa, hf, hr, draft, read, strand, anchors, ap):
    """The match list poa_realign hands poa_augment for one read (the cropped alignment, shifted
    back by the crop start)."""
    s, e = crop_range(anchors, len(draft), len(read))
    sx = draft.symbols(True, 51, s, e - s)
    sy = read.symbols(True, 51)
    a = np.asarray(anchors, dtype=np.int64).reshape(-1, 3).copy()
    a[:, 0] -= s
    m = ref_poa.align_with_indels(hf if strand else hr, sx, sy, a, ap)[0].copy()
    m[:, 1] += s
    return m


@pytest.mark.parametrize("seed,hp", [(3, False), (5, True)])
def test_node_update_equals_the_reference_graph(engine, ref_poa, ref_models, polish_model, seed, hp):
    hf, hr = ref_models
    ap = polish_model.alignment
    wl = synth.config_polish(seed=seed, n_chunks=2, chunk_len=700, coverage=12, read_len=(450, 650), hp_runs=hp)
    params_h = ref_poa.params(hf, hr, ap, max_iterations=5)
    matches = []
    for c in range(2):
        for r, s, a in zip(wl.reads[c], wl.strands[c], wl.anchors[c]):
            matches.append(_reference_matches(ref_poa, hf, hr, wl.drafts[c], r, s, a, ap))
    got = node_update(engine, wl.drafts, wl.reads, wl.strands, matches, 51, polish_model.repeat_log10)["chunks"]
    for c in range(2):
        reads_h = ref_poa.reads(wl.reads[c], wl.strands[c])
        anchors_h = ref_poa.anchors(wl.anchors[c])
        poa = ref_poa.realign(reads_h, anchors_h, wl.drafts[c], params_h)
        ref = ref_poa.nodes(poa)
        assert np.array_equal(got[c]["base_weights"], ref["base_weights"])
        assert np.array_equal(got[c]["repeat_count_weights"], ref["repeat_count_weights"])
        assert np.array_equal(got[c]["n_obs"], ref["n_obs"])
        assert np.array_equal(got[c]["observations"], ref_poa.observations(poa))
        ref_poa.estimate_repeat_counts(poa, reads_h, params_h)
        _, rc_counts = ref_poa.reference(poa)
        assert np.array_equal(got[c]["repeat_counts"], rc_counts.astype(np.uint64))
        assert (rc_counts > 1).any()
        ref_poa.free_poa(poa)
        ref_poa.free_anchors(anchors_h)
        ref_poa.free_reads(reads_h)
    ref_poa.free_params(params_h)


def _random_batch(rng, n_chunks, chunk_len, reads_per_chunk, read_len, tuples_per_read):
    bases = np.frombuffer(b"ACGT", np.uint8)
    drafts, reads, strands, matches = [], [], [], []
    for _ in range(n_chunks):
        d = bytes(bases[rng.integers(0, 4, chunk_len)])
        drafts.append(RleString(d, rng.integers(1, 8, chunk_len).astype(np.uint32)))
        lst, st = [], []
        for _ in range(reads_per_chunk):
            n = int(rng.integers(read_len // 2, read_len))
            chars = bases[rng.integers(0, 4, n)].copy()
            chars[rng.random(n) < 0.01] = ord("N")  # a few N runs: the N bin and the A table
            counts = rng.integers(1, 12, n).astype(np.uint32)
            counts[rng.random(n) < 0.02] = rng.integers(51, 70)  # over-long runs: clamped
            lst.append(RleString(bytes(chars), counts))
            st.append(int(rng.integers(0, 2)))
            k = int(rng.integers(0, tuples_per_read))
            w = rng.integers(100_000, 10_000_001, k)
            x = rng.integers(0, chunk_len, k)
            y = rng.integers(0, n, k)
            matches.append(np.stack([w, x, y], axis=1))
        reads.append(lst)
        strands.append(st)
    return drafts, reads, strands, matches


def test_node_update_equals_the_host_graph_on_large_batches(engine, polish_model):
    """Random match tuples (many per node, over-long runs, N bases, both strands) folded by the
    host graph (poa_augment with no indels) and by the GPU: identical weights, observation order
    and run lengths over 24 graphs and ~1.5 M tuples."""
    rng = np.random.default_rng(11)
    drafts, reads, strands, matches = _random_batch(rng, 24, 3000, 40, 2500, 3000)
    got = node_update(engine, drafts, reads, strands, matches, 51, polish_model.repeat_log10)["chunks"]
    host = PoaSet(None, None, polish_model.alignment, PolishParams(), drafts, reads, strands, None,
                  polish_model.repeat_log10)
    empty = np.zeros((0, 3), np.int64)
    host.realign_pairs([(m, empty, empty) for m in matches])
    for c in range(len(drafts)):
        ref = host.nodes(c)
        assert np.array_equal(got[c]["base_weights"], ref["base_weights"])
        assert np.array_equal(got[c]["repeat_count_weights"], ref["repeat_count_weights"])
        assert np.array_equal(got[c]["observations"], host.observations(c))
    host.estimate_repeat_counts()
    for c in range(len(drafts)):
        assert np.array_equal(got[c]["repeat_counts"], host.reference(c).counts.astype(np.uint64))
    host.close()
    assert sum(len(m) for m in matches) > 1_000_000


def test_node_update_without_observations_or_estimate(engine, polish_model):
    rng = np.random.default_rng(12)
    drafts, reads, strands, matches = _random_batch(rng, 3, 500, 10, 400, 300)
    full = node_update(engine, drafts, reads, strands, matches, 51, polish_model.repeat_log10)["chunks"]
    bare = node_update(engine, drafts, reads, strands, matches, 51, None, observations=False)["chunks"]
    for a, b in zip(full, bare):
        assert np.array_equal(a["base_weights"], b["base_weights"])
        assert np.array_equal(a["n_obs"], b["n_obs"])
        assert "repeat_counts" not in b and "observations" not in b


def test_node_update_rejects_tuples_outside_the_graph(engine, polish_model):
    rng = np.random.default_rng(13)
    drafts, reads, strands, matches = _random_batch(rng, 2, 200, 4, 150, 50)
    bad = [m.copy() for m in matches]
    bad[1] = np.array([[1000, len(drafts[0]), 0]])  # x = the draft's length: node past the graph
    with pytest.raises(MpError):
        node_update(engine, drafts, reads, strands, bad, 51, polish_model.repeat_log10)
    bad = [m.copy() for m in matches]
    bad[0] = np.array([[1000, 0, len(reads[0][0])]])  # y past the read
    with pytest.raises(MpError):
        node_update(engine, drafts, reads, strands, bad, 51, polish_model.repeat_log10)
    # the engine still works after a rejected batch
    ok = node_update(engine, drafts, reads, strands, matches, 51, polish_model.repeat_log10)["chunks"]
    assert len(ok) == 2
