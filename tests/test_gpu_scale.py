"""Parity at the sizes of the larger configurations (GPU against the FP64 oracle, Oracle B, and the
reference's own code, Oracle A):

* long reads at the shipped traceback schedule (minDiagsBetweenTraceBack 10000,
  traceBackDiagonals 40, impl/pairwiseAligner.c:722-793): reads of 20-100 kb at band half-width
  64 and of 100-150 kb at half-width 96, several traceback segments each;
* a slice of the batched uneven-reads workload (its first 4 chunks, homopolymer-enriched
  templates, log-normal read lengths), the reads the headline benchmark times;
* the polished consensus of one 110 kb chunk at 50x (the polishing loop at genome scale)
  against the reference's poa_realignAll run on the same chunk (golden fixture made by
  tests/golden/make_consensus_golden.py).

Oracle runs go to a thread pool (the oracles are C libraries; their calls release the GIL)."""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from marginpolish_b200 import Model, PolishParams, polish, realign_batch, synth
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


def test_consensus_of_a_110kb_chunk_identical_to_reference(engine, gmodel, polish_model):
    path = os.path.join(GOLDEN, "consensus_110kb.npz")
    if not os.path.exists(path):
        pytest.skip("consensus fixture not generated")
    import importlib.util
    spec = importlib.util.spec_from_file_location("mcg", os.path.join(GOLDEN, "make_consensus_golden.py"))
    mcg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mcg)
    z = np.load(path)
    wl = mcg.chunk_workload()
    assert mcg.digest(wl) == str(z["digest"]), "the seeded generator no longer makes the fixture's inputs"
    out = polish(engine, gmodel, polish_model, PolishParams(max_iterations=5), wl.drafts, wl.reads, wl.strands,
                 wl.anchors)
    want_chars = z["chars"].tobytes()
    want_counts = z["counts"].astype(np.uint32)
    got = out[0]
    if got.chars != want_chars or not np.array_equal(got.counts, want_counts):
        la, lb = len(got.chars), len(want_chars)
        first = next((i for i in range(min(la, lb)) if got.chars[i] != want_chars[i] or
                      got.counts[i] != want_counts[i]), min(la, lb))
        pytest.fail(f"consensus differs from the reference: {la} vs {lb} runs, first difference at run {first}")
