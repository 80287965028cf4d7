"""The bubble graph of the polish step against the reference's own impl/bubbleGraph.c (CPU).

With the shipped parameters (params/allParams.np.json: one polish iteration) the polishing loop
runs poa_polish (impl/polisher.c:2008-2031), whose bubble graph (bubbleGraph_constructFromPoa,
impl/bubbleGraph.c:800-978) is built here from a graph both sides fold from the reference
aligner's pairs, so every difference would be the bubble code's: the candidate weights over a
100-node window, the anchor nodes away from candidate variants, the read substrings between
anchors with their quality filter, the alleles (distinct read substrings, then the reference
allele) and the observation order the construction leaves in the graph. The allele scores need
the GPU (tests/test_gpu_polish.py).
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


def reference_pairs(ref_poa, hf, hr, draft, read, strand, anchors, ap):
    """What poa_realign hands poa_augment for one read (the cropping path)."""
    s, e = crop_range(anchors, len(draft), len(read))
    sx = draft.symbols(True, 51, s, e - s)
    sy = read.symbols(True, 51)
    a = np.asarray(anchors, dtype=np.int64).reshape(-1, 3).copy()
    a[:, 0] -= s
    out = []
    for lst in ref_poa.align_with_indels(hf if strand else hr, sx, sy, a, ap):
        lst = lst.copy()
        lst[:, 1] += s
        out.append(lst)
    return out


def same_bubbles(got, want):
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert (g["ref_start"], g["ref_length"]) == (w["ref_start"], w["ref_length"])
        assert len(g["alleles"]) == len(w["alleles"])
        for (gc, gn), (wc, wn) in zip(g["alleles"], w["alleles"]):
            assert gc == wc and np.array_equal(gn, wn)
        assert np.array_equal(g["reads"], w["reads"])
        assert np.array_equal(g["quals"], w["quals"])


def build_both(ref_poa, ref_models, polish_model, wl, quals, pp):
    """Our graph from the reference pairs, and the reference's own poa_realign, per chunk."""
    hf, hr = ref_models
    ap = polish_model.alignment
    pairs = []
    for c in range(len(wl.drafts)):
        for r, s, a in zip(wl.reads[c], wl.strands[c], wl.anchors[c]):
            pairs.append(reference_pairs(ref_poa, hf, hr, wl.drafts[c], r, s, a, ap))
    ours = PoaSet(None, None, ap, pp, wl.drafts, wl.reads, wl.strands, wl.anchors, polish_model.repeat_log10,
                  qualities=quals)
    ours.realign_pairs(pairs)
    params_h = ref_poa.params(hf, hr, ap, max_iterations=pp.max_iterations)
    ref_poa.set_polish(params_h, pp)
    refs = []
    for c in range(len(wl.drafts)):
        reads_h = ref_poa.reads(wl.reads[c], wl.strands[c])
        if quals is not None:
            ref_poa.set_qualities(reads_h, quals[c])
        anchors_h = ref_poa.anchors(wl.anchors[c])
        poa = ref_poa.realign(reads_h, anchors_h, wl.drafts[c], params_h)
        refs.append((reads_h, anchors_h, poa))
    return ours, params_h, refs


def free_refs(ref_poa, params_h, refs):
    for reads_h, anchors_h, poa in refs:
        ref_poa.free_poa(poa)
        ref_poa.free_anchors(anchors_h)
        ref_poa.free_reads(reads_h)
    ref_poa.free_params(params_h)


@pytest.mark.parametrize("seed,hp,coverage,with_quals", [(3, False, 12, False), (5, True, 24, True),
                                                         (9, True, 30, True)])
def test_bubble_graph_identical_to_reference(ref_poa, ref_models, polish_model, seed, hp, coverage, with_quals):
    wl = synth.config_polish(seed=seed, n_chunks=2, chunk_len=700, coverage=coverage, read_len=(450, 650),
                             hp_runs=hp)
    quals = wl.qualities(seed) if with_quals else None
    pp = PolishParams.shipped()
    ours, params_h, refs = build_both(ref_poa, ref_models, polish_model, wl, quals, pp)
    ours.build_bubbles()
    n_bubbles = 0
    filtered = 0
    for c, (reads_h, _, poa) in enumerate(refs):
        want = ref_poa.bubble_graph(poa, reads_h, params_h)
        got = ours.bubbles(c)
        same_bubbles(got, want["bubbles"])
        # the construction sorts every node's observations (by read, then descending weight)
        assert np.array_equal(ours.observations(c), ref_poa.observations(poa))
        n_bubbles += len(got)
        for b in got:
            assert len(b["alleles"]) > 1 and b["reads"].shape[0] > 0
            if with_quals and b["reads"].shape[0] == pp.filter_reads_coverage:
                filtered += 1
    assert n_bubbles > 0
    if with_quals and coverage > pp.filter_reads_coverage:
        assert filtered > 0  # some bubbles lost low-quality substrings to the filter
    ours.close()
    free_refs(ref_poa, params_h, refs)


def test_polish_refuses_the_unbuilt_allele_source(polish_model):
    wl = synth.config_polish(seed=7, n_chunks=1, chunk_len=300, coverage=4, read_len=(200, 280))
    pp = PolishParams.shipped()
    pp.use_read_alleles = False
    from marginpolish_b200._lib import MpError
    with pytest.raises(MpError) as err:
        PoaSet(None, None, polish_model.alignment, pp, wl.drafts, wl.reads, wl.strands, wl.anchors,
               polish_model.repeat_log10)
    assert "not built" in str(err.value)


def test_bubble_scoring_needs_an_engine(ref_poa, ref_models, polish_model):
    wl = synth.config_polish(seed=3, n_chunks=1, chunk_len=500, coverage=10, read_len=(300, 450))
    pp = PolishParams.shipped()
    ours, params_h, refs = build_both(ref_poa, ref_models, polish_model, wl, None, pp)
    ours.build_bubbles()
    from marginpolish_b200._lib import MpError
    with pytest.raises(MpError):
        ours.score_bubbles()
    with pytest.raises(MpError):
        ours.bubble_consensus(0)  # not scored
    ours.close()
    free_refs(ref_poa, params_h, refs)
