"""The POA steps of the polishing loop against the reference's own impl/polisher.c (CPU).

The library's graph is built from the reference aligner's pairs (the cropping path of
getAlignedPairsWithIndelsCroppingReference, impl/polisher.c:605-654), so every difference
would be the POA code's: node base and run-length weights, observation lists (in order),
inserts and deletes with their strings, weights and observations (poa_augment,
:316-534), the consensus and its node map (poa_getConsensus, :1025-1275), the next anchors
(poa_getAnchorAlignments, :536-592), the run-length estimate (:1556-1565, :1756-1865) and
the stop rule's score (:709-758) must all be identical.
"""
import os

import numpy as np
import pytest

from marginpolish_b200 import PoaSet, PolishParams, synth
from marginpolish_b200.rle import crop_range

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


def _reference_pairs(ref_poa, hf, hr, draft, read, strand, anchors, ap):
    """What poa_realign hands poa_augment for one read: the crop, the aligner on the cropped
    symbols, the pairs shifted back by the crop start."""
    s, e = crop_range(anchors, len(draft), len(read))
    sx = draft.symbols(True, 51, s, e - s)
    sy = read.symbols(True, 51)
    a = np.asarray(anchors, dtype=np.int64).reshape(-1, 3).copy()
    a[:, 0] -= s
    lists = ref_poa.align_with_indels(hf if strand else hr, sx, sy, a, ap)
    out = []
    for lst in lists:
        lst = lst.copy()
        lst[:, 1] += s
        out.append(lst)
    return out  # (matches, gap-x, gap-y)


@pytest.mark.parametrize("seed,hp", [(3, False), (5, True)])
def test_poa_steps_identical_to_reference(ref_poa, ref_models, polish_model, seed, hp):
    hf, hr = ref_models
    ap = polish_model.alignment
    wl = synth.config_polish(seed=seed, n_chunks=2, chunk_len=700, coverage=12, read_len=(450, 650), hp_runs=hp)
    pp = PolishParams(max_iterations=5)
    params_h = ref_poa.params(hf, hr, ap, max_iterations=5)
    pairs = []
    for c in range(2):
        for r, s, a in zip(wl.reads[c], wl.strands[c], wl.anchors[c]):
            pairs.append(_reference_pairs(ref_poa, hf, hr, wl.drafts[c], r, s, a, ap))
    ours = PoaSet(None, None, ap, pp, wl.drafts, wl.reads, wl.strands, wl.anchors, polish_model.repeat_log10)
    ours.realign_pairs(pairs)
    for c in range(2):
        reads_h = ref_poa.reads(wl.reads[c], wl.strands[c])
        anchors_h = ref_poa.anchors(wl.anchors[c])
        poa = ref_poa.realign(reads_h, anchors_h, wl.drafts[c], params_h)
        # the graph (poa_realign / poa_augment)
        a, b = ours.nodes(c), ref_poa.nodes(poa)
        assert a["bases"] == b["bases"]
        for k in ("repeat_counts", "base_weights", "repeat_count_weights", "n_obs", "n_ins", "n_del"):
            assert np.array_equal(a[k], b[k]), k
        assert np.array_equal(ours.observations(c), ref_poa.observations(poa))
        assert ours.inserts(c) == ref_poa.inserts(poa)
        assert ours.deletes(c) == ref_poa.deletes(poa)
        assert ours.info(c)["score"] == ref_poa.score(poa)
        assert len(ours.inserts(c)) > 0 and len(ours.deletes(c)) > 0
        # the consensus walk and the next anchors
        cons, node_map = ours.consensus(c)
        rchars, rcounts, rmap = ref_poa.consensus(poa, params_h)
        assert cons.chars == rchars and np.array_equal(cons.counts, rcounts.astype(np.uint32))
        assert np.array_equal(node_map, rmap)
        assert cons.chars != wl.drafts[c].chars or not np.array_equal(cons.counts, wl.drafts[c].counts)
        ours_a = ours.anchor_alignments(c, node_map)
        ref_a = ref_poa.anchor_alignments(poa, rmap, len(wl.reads[c]), params_h)
        assert all(np.array_equal(x, y) for x, y in zip(ours_a, ref_a))
        ref_poa.estimate_repeat_counts(poa, reads_h, params_h)
        rc_chars, rc_counts = ref_poa.reference(poa)
        ref_poa.free_poa(poa)
        ref_poa.free_anchors(anchors_h)
        ref_poa.free_reads(reads_h)
        pending = (rc_chars, rc_counts)
        if c == 0:
            first = pending
        else:
            second = pending
    # run-length estimate of both chunks at once
    ours.estimate_repeat_counts()
    for c, (rc_chars, rc_counts) in enumerate((first, second)):
        got = ours.reference(c)
        assert got.chars == rc_chars and np.array_equal(got.counts, rc_counts.astype(np.uint32))
    ours.close()
    ref_poa.free_params(params_h)


def test_realign_needs_an_engine(polish_model):
    wl = synth.config_polish(seed=7, n_chunks=1, chunk_len=300, coverage=4, read_len=(200, 280))
    s = PoaSet(None, None, polish_model.alignment, PolishParams(), wl.drafts, wl.reads, wl.strands, wl.anchors,
               polish_model.repeat_log10)
    from marginpolish_b200._lib import MpError
    with pytest.raises(MpError):
        s.realign()
    with pytest.raises(MpError):
        s.consensus(0)  # no graph yet
    s.close()


def test_device_steps_flags_and_node_update_arguments(polish_model):
    """mp_poa_set_device_steps takes only its two step bits; mp_node_update refuses a missing
    engine or batch before it touches a GPU."""
    import ctypes

    from marginpolish_b200 import _lib
    from marginpolish_b200._lib import MpError
    wl = synth.config_polish(seed=8, n_chunks=1, chunk_len=300, coverage=4, read_len=(200, 280))
    s = PoaSet(None, None, polish_model.alignment, PolishParams(), wl.drafts, wl.reads, wl.strands, wl.anchors,
               polish_model.repeat_log10)
    s.set_device_steps(run_lengths=False, indels=False)
    s.set_device_steps()
    lib = _lib.load()
    assert lib.mp_poa_set_device_steps(s.handle, 4) == _lib.MP_ERR_ARGUMENT
    s.close()
    r = _lib.NodeResult()
    assert lib.mp_node_update(None, None, ctypes.byref(r)) == _lib.MP_ERR_ARGUMENT
    with pytest.raises(MpError):
        _lib.check(lib.mp_node_update(None, None, ctypes.byref(r)))
