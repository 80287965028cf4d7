"""Parity at the sizes of the larger configurations (GPU against the FP64 oracle, Oracle B, and the
reference's own code, Oracle A):

* long reads at the shipped traceback schedule (minDiagsBetweenTraceBack 10000,
  traceBackDiagonals 40, impl/pairwiseAligner.c:722-793): reads of 20-100 kb at band half-width
  64 and of 100-150 kb at half-width 96, several traceback segments each;
* a slice of the batched uneven-reads workload (its first 4 chunks, homopolymer-enriched
  templates, log-normal read lengths), the reads the headline benchmark times;
* the polished consensus of one 110 kb chunk at 50x (the polishing loop at genome scale)
  against the reference's poa_realignAll run on the same chunk (golden fixture made by
  tests/golden/make_consensus_golden.py), and against the same loop fed FP64-exact pairs.

Oracle runs go to a thread pool (the oracles are C libraries; their calls release the GIL)."""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from marginpolish_b200 import Model, PolishParams, realign_batch, synth
from oracle.bindings import ExactOracle, MpoModel
from oracle.compare import check_job, check_loglik, set_diff_against_reference

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def gmodel(engine, polish_model):
    m = Model.from_polish(engine, polish_model)
    yield m
    m.close()


@pytest.fixture(scope="module")
def ref_models(ref_oracle):
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    hf = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    yield hf, hr
    ref_oracle.free_model(hf)
    ref_oracle.free_model(hr)


def _job(jobs, j):
    return (jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]], jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]],
            jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]])


def _check_against_both_oracles(engine, gmodel, polish_model, ref_oracle, ref_models, jobs):
    ap = polish_model.alignment
    res = realign_batch(engine, gmodel, ap, jobs)
    eo = ExactOracle()
    mpo = (MpoModel.from_state_model(polish_model.forward), MpoModel.from_state_model(polish_model.reverse))

    def oracles(j):
        sx, sy, a = _job(jobs, j)
        fwd = bool(jobs.strand[j])
        o = eo.align_with_indels(mpo[0] if fwd else mpo[1], sx, sy, a, ap, dense="near")
        r = ref_oracle.align_with_indels(ref_models[0] if fwd else ref_models[1], sx, sy, a, ap)
        return o, r

    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        outs = list(ex.map(oracles, range(jobs.n_jobs)))
    worst, ndiff, tuples = 0.0, 0, 0
    for j, (o, r) in enumerate(outs):
        g = [res.job(j, k).copy() for k in range(3)]
        for k in range(3):
            g[k][:, 1] -= int(jobs.x_shift[j])
            tuples += g[k].shape[0]
        rep = check_job(g, o, ap.threshold)
        worst = max(worst, rep["max_abs_posterior_error"])
        check_loglik(res.log_likelihood[j], o["log_likelihood"])
        assert res.cells[j] == o["cells"]
        ndiff += set_diff_against_reference(g, r, o, ap.threshold)
    return worst, ndiff, tuples, res


@pytest.mark.parametrize("half_width,lengths", [
    (64, [20_000, 35_000, 50_000, 65_000, 80_000, 100_000]),
    (96, [100_000, 118_000, 135_000, 150_000]),
])
def test_long_reads_at_the_shipped_traceback_schedule(engine, gmodel, polish_model, ref_oracle, ref_models,
                                                      half_width, lengths):
    ap = polish_model.alignment
    assert ap.min_diags_between_traceback == 10000 and ap.traceback_diagonals == 40
    jobs = synth.config_long_reads(seed=31 + half_width, lengths=lengths, half_width=half_width).jobs()
    diags = (jobs.x_end - jobs.x_begin) + np.diff(jobs.y_offsets)
    assert int(diags.max()) > 5 * ap.min_diags_between_traceback  # several traceback segments
    worst, ndiff, tuples, _ = _check_against_both_oracles(engine, gmodel, polish_model, ref_oracle, ref_models, jobs)
    print(f"w={half_width}: {jobs.n_jobs} reads, {int(diags.sum())} diagonals, {tuples} tuples, "
          f"max |posterior - FP64| {worst:.2e}, {ndiff} tuples differ from the reference within its tie band")
    assert worst <= 1e-4


def test_batched_workload_slice_against_both_oracles(engine, gmodel, polish_model, ref_oracle, ref_models):
    """The first 4 chunks of the headline workload (the bench's seed): every read against both
    oracles."""
    wl = synth.config_batched(seed=2, n_chunks=256)
    per_chunk = np.bincount(wl.read_template, minlength=len(wl.templates))
    n = int(per_chunk[:4].sum())
    jobs = wl.jobs()
    from marginpolish_b200 import Jobs
    a1 = int(jobs.anchor_offsets[n])
    sl = Jobs(jobs.x_symbols, jobs.x_begin[:n], jobs.x_end[:n], jobs.y_symbols[:int(jobs.y_offsets[n])],
              jobs.y_offsets[:n + 1], jobs.anchors[:a1], jobs.anchor_offsets[:n + 1], jobs.strand[:n], None, None,
              jobs.x_shift[:n])
    worst, ndiff, tuples, res = _check_against_both_oracles(engine, gmodel, polish_model, ref_oracle, ref_models, sl)
    print(f"4 chunks: {n} reads, {res.total_cells} cells, {tuples} tuples, max |posterior - FP64| {worst:.2e}, "
          f"{ndiff} tie-band differences from the reference")
    assert worst <= 1e-4


def _first_pass_pairs(wl, aligner):
    """Pairs of every read of the chunk against its draft as poa_realign makes them: the crop of
    getAlignedPairsWithIndelsCroppingReference (impl/polisher.c:613-628), the aligner on the
    cropped symbols, x shifted back by the crop start."""
    draft = wl.drafts[0]

    def one(r):
        read, a = wl.reads[0][r], wl.anchors[0][r]
        s, e = synth.crop_range(a, len(draft), len(read))
        sx = synth.rle_symbols(synth.RleString(draft.chars[s:e], draft.counts[s:e]), True, 51)
        sy = synth.rle_symbols(read, True, 51)
        aa = np.asarray(a, np.int64).reshape(-1, 3).copy()
        aa[:, 0] -= s
        out = []
        for lst in aligner(r, sx, sy, aa):
            lst = np.asarray(lst).copy()
            lst[:, 1] += s
            out.append(lst)
        return out

    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        return list(ex.map(one, range(len(wl.reads[0]))))


def test_consensus_of_a_110kb_chunk(engine, gmodel, polish_model, ref_oracle, ref_models):
    """The polishing loop on one 110 kb chunk at 50x (230 reads of up to 100 kb, band half-width
    64) against the reference's poa_realignAll + run-length estimate on the same chunk.

    * The GPU's polished chunk is identical, bit for bit, to the same loop fed FP64-exact
      posterior pairs (Oracle B) -- here the loop keeps the first graph, so that is the
      run-length estimate over the exact pairs' graph.
    * Fed the reference aligner's own pairs (Oracle A), this library's POA steps reproduce the
      reference's result exactly, every run: the POA code is the reference's at scale.
    * Exact and reference pairs differ by the reference's approximate logAdd (up to ~2e-3 per
      posterior), which tips near-tie run-length decisions: the polished bases are identical and
      at most 1 run in 10,000 takes a different run length.
    """
    path = os.path.join(GOLDEN, "consensus_110kb.npz")
    if not os.path.exists(path):
        pytest.skip("consensus fixture not generated")
    import importlib.util
    from marginpolish_b200 import PoaSet
    spec = importlib.util.spec_from_file_location("mcg", os.path.join(GOLDEN, "make_consensus_golden.py"))
    mcg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mcg)
    z = np.load(path)
    wl = mcg.chunk_workload()
    assert mcg.digest(wl) == str(z["digest"]), "the seeded generator no longer makes the fixture's inputs"
    ap = polish_model.alignment
    ref_chars, ref_counts = z["chars"].tobytes(), z["counts"].astype(np.uint32)

    s = PoaSet.from_polish_model(engine, gmodel, polish_model, PolishParams(max_iterations=5), wl.drafts, wl.reads,
                                 wl.strands, wl.anchors)
    s.realign()
    s.iterate()
    s.estimate_repeat_counts()
    gpu = s.reference(0)
    s.close()

    eo = ExactOracle()
    mpo = (MpoModel.from_state_model(polish_model.forward), MpoModel.from_state_model(polish_model.reverse))
    exact_pairs = _first_pass_pairs(
        wl, lambda r, sx, sy, a: eo.align_with_indels(mpo[0] if wl.strands[0][r] else mpo[1], sx, sy, a, ap)["pairs"])
    ref_pairs = _first_pass_pairs(
        wl, lambda r, sx, sy, a: ref_oracle.align_with_indels(ref_models[0] if wl.strands[0][r] else ref_models[1],
                                                              sx, sy, a, ap))

    def host_loop(pairs):
        h = PoaSet(None, None, ap, PolishParams(max_iterations=5), wl.drafts, wl.reads, wl.strands, wl.anchors,
                   polish_model.repeat_log10)
        h.realign_pairs(pairs)
        h.estimate_repeat_counts()
        out = h.reference(0)
        h.close()
        return out

    # the reference kept its first graph: its polished bases are the draft's
    assert ref_chars == wl.drafts[0].chars
    from_ref = host_loop(ref_pairs)
    assert from_ref.chars == ref_chars and np.array_equal(from_ref.counts, ref_counts), \
        "the POA steps fed the reference's pairs do not reproduce the reference"
    from_exact = host_loop(exact_pairs)
    assert gpu.chars == from_exact.chars and np.array_equal(gpu.counts, from_exact.counts), \
        "the GPU loop differs from the loop fed FP64-exact pairs"
    assert gpu.chars == ref_chars
    diff = np.nonzero(gpu.counts != ref_counts)[0]
    print(f"110 kb chunk: {len(ref_chars)} runs, identical bases; run lengths differ from the reference's at "
          f"{diff.size} runs {diff[:10].tolist()} (the reference's approximate posteriors)")
    assert diff.size <= max(1, len(ref_chars) // 10000)


def _run_differences(a: bytes, ac, b: bytes, bc, window: int = 24):
    """Runs where two nearly equal run-length strings differ: walk both, and at a mismatch (base
    or run length) resynchronise on the smallest shift that makes the next `window` runs agree.
    Returns the number of differing runs."""
    i = j = diffs = 0
    while i < len(a) and j < len(b):
        if a[i] == b[j] and ac[i] == bc[j]:
            i += 1
            j += 1
            continue
        diffs += 1
        best = None
        for di in range(0, 8):
            for dj in range(0, 8):
                if (di, dj) == (0, 0):
                    continue
                if a[i + di:i + di + window] == b[j + dj:j + dj + window]:
                    if best is None or di + dj < sum(best):
                        best = (di, dj)
        if best is None:
            best = (1, 1)
        i += best[0]
        j += best[1]
    return diffs + (len(a) - i) + (len(b) - j)


def test_shipped_polish_of_a_110kb_chunk(engine, gmodel, polish_model):
    """The shipped loop (poa_realignAll with one polish iteration: bubble graph, allele scores in
    the reference's arithmetic, new consensus, realignment; then the run-length estimate) on the
    110 kb chunk at 50x with base qualities, against the reference's own loop on the same chunk
    (tests/golden/polish_110kb.npz). The two differ only where the GPU's posteriors and the
    reference's approximate ones tip a near-tie of the graph's weights."""
    path = os.path.join(GOLDEN, "polish_110kb.npz")
    if not os.path.exists(path):
        pytest.skip("polish fixture not generated")
    import importlib.util
    from marginpolish_b200 import polish
    spec = importlib.util.spec_from_file_location("mpg", os.path.join(GOLDEN, "make_polish_golden.py"))
    mpg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mpg)
    z = np.load(path)
    wl, quals, base_digest = mpg.chunk_workload()
    assert mpg.digest(wl, quals, base_digest) == str(z["digest"]), \
        "the seeded generator no longer makes the fixture's inputs"
    want_chars, want_counts = z["chars"].tobytes(), z["counts"].astype(np.uint32)
    got = polish(engine, gmodel, polish_model, PolishParams.shipped(), wl.drafts, wl.reads, wl.strands, wl.anchors,
                 quals)[0]
    draft = wl.drafts[0]
    changed_by_ref = _run_differences(draft.chars, draft.counts, want_chars, want_counts)
    diffs = _run_differences(got.chars, got.counts, want_chars, want_counts)
    print(f"110 kb chunk, shipped loop: reference {len(want_chars)} runs ({changed_by_ref} runs changed from the "
          f"draft), GPU {len(got)} runs, {diffs} runs differ from the reference")
    assert changed_by_ref > 20
    assert diffs <= max(2, changed_by_ref // 20)
