"""The polish step on the GPU (poa_polish, impl/polisher.c:2008-2031, with the bubble graph of
impl/bubbleGraph.c:800-978) against the reference's own code.

* mp_forward_pairs computes computeForwardProbability (impl/pairwiseAligner.c:813-865) in the
  reference's arithmetic: every pair's log-likelihood equals the reference's bit for bit, for
  alleles of every length class (shared-memory rows of 16, 32 and 64 runs, global-memory rows
  beyond) and both strands.
* Built from the reference aligner's pairs, the bubble graph's allele supports (float, as the
  reference stores them), the chosen alleles, the new consensus and its map equal the
  reference's.
* The whole shipped loop (poa_realignAll with one polish iteration, then the run-length
  estimate) fed the reference aligner's pairs reproduces the reference's polished chunk exactly;
  with the GPU's own posterior pass it differs only where the reference's approximate
  posteriors tip a near-tie.
"""
import os

import numpy as np
import pytest

from marginpolish_b200 import Model, PoaSet, PolishParams, forward_pairs, forward_pairs_timing, polish, synth

from test_poa_bubbles_host import build_both, free_refs, reference_pairs, same_bubbles

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def gmodel(engine, polish_model):
    m = Model.from_polish(engine, polish_model)
    yield m
    m.close()


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


def _rle_symbols(rng, n):
    b = rng.integers(0, 4, size=n)
    c = rng.integers(1, 51, size=n)
    c[rng.random(n) < 0.7] = 1  # mostly short runs, as in reads
    return ((c << 8) | b).astype(np.uint16)


def test_pair_scores_bit_exact_with_reference(engine, gmodel, polish_model, ref_oracle):
    """Every length class and both strands; alleles and read substrings shared between pairs."""
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    hf = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    rng = np.random.default_rng(11)
    ap = polish_model.alignment
    lengths = [0, 1, 2, 7, 16, 17, 31, 32, 33, 50, 64, 65, 90, 140]
    xs_list = [_rle_symbols(rng, n) for n in lengths]
    ys_list = [_rle_symbols(rng, n) for n in lengths]
    x_sym = np.concatenate(xs_list)
    y_sym = np.concatenate(ys_list)
    x_off = np.concatenate([[0], np.cumsum(lengths)[:-1]])
    y_off = x_off.copy()
    pairs = [(i, j, s) for i in range(len(lengths)) for j in range(len(lengths)) for s in (0, 1)
             if (i + j + s) % 3 != 1 or lengths[i] > 60]
    xo = np.array([x_off[i] for i, _, _ in pairs])
    xl = np.array([lengths[i] for i, _, _ in pairs])
    yo = np.array([y_off[j] for _, j, _ in pairs])
    yl = np.array([lengths[j] for _, j, _ in pairs])
    st = np.array([s for _, _, s in pairs])
    got = forward_pairs(engine, gmodel, x_sym, y_sym, xo, xl, yo, yl, st)
    for k, (i, j, s) in enumerate(pairs):
        want = ref_oracle.forward_probability(hf if s else hr, xs_list[i], ys_list[j], np.zeros((0, 3)), ap)
        assert got[k] == want, (lengths[i], lengths[j], s, got[k], want)
    assert len(pairs) > 250
    t = forward_pairs_timing(engine)
    assert t["pairs"] == len(pairs) and t["cells"] == int(np.sum((xl + 1) * (yl + 1)))
    ref_oracle.free_model(hf)
    ref_oracle.free_model(hr)


def test_pair_scores_refuse_out_of_table_run_lengths(engine, gmodel):
    from marginpolish_b200._lib import MpError
    x = np.array([(51 << 8) | 2], np.uint16)
    y = np.array([(1 << 8) | 2], np.uint16)
    with pytest.raises(MpError):
        forward_pairs(engine, gmodel, x, y, [0], [1], [0], [1], [1])
    with pytest.raises(MpError):
        forward_pairs(engine, gmodel, x, y, [0], [2], [0], [1], [1])  # outside the buffer


@pytest.mark.parametrize("seed,hp,coverage,with_quals", [(3, False, 12, False), (5, True, 24, True),
                                                         (9, True, 30, True)])
def test_bubble_supports_and_consensus_identical_to_reference(engine, gmodel, ref_poa, ref_models, polish_model,
                                                              seed, hp, coverage, with_quals):
    wl = synth.config_polish(seed=seed, n_chunks=2, chunk_len=700, coverage=coverage, read_len=(450, 650),
                             hp_runs=hp)
    quals = wl.qualities(seed) if with_quals else None
    pp = PolishParams.shipped()
    host, params_h, refs = build_both(ref_poa, ref_models, polish_model, wl, quals, pp)
    host.close()
    # the same graph in a set with the engine, so that the scores run on the GPU
    ours = PoaSet(engine, gmodel, polish_model.alignment, pp, wl.drafts, wl.reads, wl.strands, wl.anchors,
                  polish_model.repeat_log10, qualities=quals)
    hf, hr = ref_models
    ours.realign_pairs([reference_pairs(ref_poa, hf, hr, wl.drafts[c], r, s, a, polish_model.alignment)
                        for c in range(2) for r, s, a in zip(wl.reads[c], wl.strands[c], wl.anchors[c])])
    ours.build_bubbles()
    ours.score_bubbles()
    changed = 0
    for c, (reads_h, _, poa) in enumerate(refs):
        want = ref_poa.bubble_graph(poa, reads_h, params_h)
        got = ours.bubbles(c)
        same_bubbles(got, want["bubbles"])
        for g, w in zip(got, want["bubbles"]):
            assert np.array_equal(g["supports"], w["supports"])  # float32, bit for bit
        path, cons, node_map = ours.bubble_consensus(c)
        assert np.array_equal(path, want["path"])
        assert cons.chars == want["chars"] and np.array_equal(cons.counts, want["counts"].astype(np.uint32))
        assert np.array_equal(node_map, want["map"])
        changed += int(cons.chars != wl.drafts[c].chars or not np.array_equal(cons.counts, wl.drafts[c].counts))
    assert changed > 0  # the polish step changed at least one chunk
    ours.close()
    free_refs(ref_poa, params_h, refs)


def _pairs_against(ref_poa, models, ap, consensus, reads, strands, anchors):
    return [reference_pairs(ref_poa, models[0], models[1], consensus, r, s, a, ap)
            for r, s, a in zip(reads, strands, anchors)]


def test_shipped_loop_identical_to_reference(engine, gmodel, ref_poa, ref_models, polish_model):
    """poa_realignAll with the shipped parameters (no consensus iterations, one polish iteration),
    then the run-length estimate (marginPolish.c:554-560), on two homopolymer-rich chunks with
    qualities. Fed the reference aligner's pairs at both realignments, the library's loop gives
    the reference's polished chunks exactly; the GPU loop differs from them only where the
    reference's approximate posteriors tip a near-tie."""
    ap = polish_model.alignment
    hf, hr = ref_models
    wl = synth.config_polish(seed=31, n_chunks=2, chunk_len=1500, coverage=24, read_len=(900, 1400), hp_runs=True)
    quals = wl.qualities(31)
    pp = PolishParams.shipped()
    params_h = ref_poa.params(hf, hr, ap, max_iterations=0)
    ref_poa.set_polish(params_h, pp)
    want = []
    for c in range(2):
        reads_h = ref_poa.reads(wl.reads[c], wl.strands[c])
        ref_poa.set_qualities(reads_h, quals[c])
        anchors_h = ref_poa.anchors(wl.anchors[c])
        poa = ref_poa.realign_all(reads_h, anchors_h, wl.drafts[c], params_h)
        ref_poa.estimate_repeat_counts(poa, reads_h, params_h)
        want.append(ref_poa.reference(poa))
        ref_poa.free_poa(poa)
        ref_poa.free_anchors(anchors_h)
        ref_poa.free_reads(reads_h)
    ref_poa.free_params(params_h)

    # the library's steps fed the reference aligner's pairs
    for c in range(2):
        s1 = PoaSet(engine, gmodel, ap, pp, [wl.drafts[c]], [wl.reads[c]], [wl.strands[c]], [wl.anchors[c]],
                    polish_model.repeat_log10, qualities=[quals[c]])
        s1.realign_pairs(_pairs_against(ref_poa, (hf, hr), ap, wl.drafts[c], wl.reads[c], wl.strands[c],
                                            wl.anchors[c]))
        s1.build_bubbles()
        s1.score_bubbles()
        _, cons, node_map = s1.bubble_consensus(0)
        if cons.chars == wl.drafts[c].chars and np.array_equal(cons.counts, wl.drafts[c].counts):
            s1.estimate_repeat_counts()
            got = s1.reference(0)
        else:
            anchors2 = s1.anchor_alignments(0, node_map)
            s2 = PoaSet(None, None, ap, pp, [cons], [wl.reads[c]], [wl.strands[c]], [anchors2],
                        polish_model.repeat_log10, qualities=[quals[c]])
            s2.realign_pairs(_pairs_against(ref_poa, (hf, hr), ap, cons, wl.reads[c], wl.strands[c], anchors2))
            s2.estimate_repeat_counts()
            got = s2.reference(0)
            s2.close()
        s1.close()
        assert got.chars == want[c][0] and np.array_equal(got.counts, want[c][1].astype(np.uint32)), c
        assert got.chars != wl.drafts[c].chars  # the polish step changed the chunk

    # the GPU loop end to end
    gpu = polish(engine, gmodel, polish_model, pp, wl.drafts, wl.reads, wl.strands, wl.anchors, quals)
    for c in range(2):
        same = gpu[c].chars == want[c][0] and np.array_equal(gpu[c].counts, want[c][1].astype(np.uint32))
        if not same:
            from difflib import SequenceMatcher
            ratio = SequenceMatcher(None, gpu[c].chars, want[c][0]).ratio()
            print(f"chunk {c}: GPU loop differs from the reference ({len(gpu[c])} vs {len(want[c][0])} runs, "
                  f"similarity {ratio:.5f})")
            assert ratio > 0.999


def _rle_list(z, name, off_name=None):
    off = z[(off_name or name) + "_offsets"]
    chars = z[name + "_chars"].tobytes()
    counts = z[name + "_counts"].astype(np.uint32)
    from marginpolish_b200.rle import RleString as R
    return [R(chars[off[i]:off[i + 1]], counts[off[i]:off[i + 1]]) for i in range(off.size - 1)]


def _identity(a: str, b: str) -> float:
    """2 * matches / (len a + len b) of a global alignment (unit edit costs)."""
    from difflib import SequenceMatcher
    m = sum(blk.size for blk in SequenceMatcher(None, a, b, autojunk=False).get_matching_blocks())
    return 2.0 * m / (len(a) + len(b))


def test_real_nanopore_windows_identical_to_reference(engine, gmodel, polish_model):
    """Real reads: the reference's own polishing examples (20 E. coli windows of Guppy-called
    nanopore reads, tests/polisherTest.c:736-819), polished without anchors with the test's loop
    (up to 100 consensus iterations at reference base penalty 0.6, then three polish
    iterations) and the run-length estimate. The GPU loop gives the reference's polished windows
    exactly (tests/golden/ecoli_windows.npz, made by make_ecoli_golden.py), and moves them
    towards the true reference."""
    path = os.path.join(GOLDEN, "ecoli_windows.npz")
    z = np.load(path)
    import importlib.util
    spec = importlib.util.spec_from_file_location("meg", os.path.join(GOLDEN, "make_ecoli_golden.py"))
    meg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(meg)
    drafts = _rle_list(z, "draft")
    truths = _rle_list(z, "truth")
    want = _rle_list(z, "polished")
    flat_reads = _rle_list(z, "read")
    cr = z["chunk_reads"]
    reads = [flat_reads[cr[w]:cr[w + 1]] for w in range(cr.size - 1)]
    strands = [list(z["strands"][cr[w]:cr[w + 1]]) for w in range(cr.size - 1)]
    got = polish(engine, gmodel, polish_model, meg.loop_params(), drafts, reads, strands, None)
    same = [g.chars == w.chars and np.array_equal(g.counts, w.counts) for g, w in zip(got, want)]
    before = sum(_identity(d.expand(), t.expand()) for d, t in zip(drafts, truths)) / len(drafts)
    after = sum(_identity(g.expand(), t.expand()) for g, t in zip(got, truths)) / len(got)
    print(f"{len(got)} E. coli windows, {len(flat_reads)} reads: {sum(same)} identical to the reference's polished "
          f"windows; identity to the truth {before:.4f} -> {after:.4f}")
    assert all(same)
    assert after > before
