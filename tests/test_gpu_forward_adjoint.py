"""GPU parity of the forward-likelihood and adjoint entry points.

* mp_forward_batch (computeForwardProbability, impl/pairwiseAligner.c:813-865) against
  the FP64 oracle on the same band (band_construct), anchored reads and anchor-free
  bubble-graph-sized pairs (impl/bubbleGraph.c:924), ragged ends, empty sequences;
  tolerance 1e-5 relative on ln P (FP32 scaled probabilities);
* mp_expectations_batch against the FP64 oracle's expected counts (relative 1e-4 on
  counts above 1, absolute 1e-4 below) and against central finite differences of the
  FP64 log-likelihood (the gradient the counts stand for);
* the transition counts against the reference's own getExpectationsUsingAnchors within
  the error of its approximate logAdd (2e-3).
"""
import numpy as np
import pytest

from marginpolish_b200 import Jobs, Model, expectations_batch, forward_batch, synth
from oracle.bindings import MpoModel

pytestmark = pytest.mark.gpu


def _job(jobs, j):
    sx = jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]]
    sy = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
    a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
    return sx, sy, a


def _rle(rng, n):
    b = rng.integers(0, 4, size=n)
    c = rng.integers(1, 6, size=n)
    return ((c << 8) | b).astype(np.uint16)


@pytest.fixture(scope="module")
def gmodel(engine, polish_model):
    m = Model.from_polish(engine, polish_model)
    yield m
    m.close()


def _ll_close(got, want):
    assert abs(got - want) <= 1e-5 * max(1.0, abs(want)), (got, want)


def test_forward_anchored_reads(engine, gmodel, polish_model, exact_oracle):
    ap = polish_model.alignment
    jobs = synth.config_small(seed=11, n_reads=6).jobs()
    rl = np.array([0, 1, 0, 1, 0, 0], np.uint8)
    rr = np.array([0, 0, 1, 1, 0, 1], np.uint8)
    jobs = Jobs(jobs.x_symbols, jobs.x_begin, jobs.x_end, jobs.y_symbols, jobs.y_offsets, jobs.anchors,
                jobs.anchor_offsets, jobs.strand, rl, rr)
    got = forward_batch(engine, gmodel, ap, jobs)
    for j in range(jobs.n_jobs):
        sx, sy, a = _job(jobs, j)
        m = MpoModel.from_state_model(polish_model.forward if jobs.strand[j] else polish_model.reverse)
        want = exact_oracle.forward_probability(m, sx, sy, a, ap.diagonal_expansion, False, bool(rl[j]), bool(rr[j]))
        _ll_close(got[j], want)


def test_forward_anchor_free_pairs(engine, gmodel, polish_model, exact_oracle):
    """The bubble graph's calls: allele vs read substring, no anchors (the band is the matrix)."""
    ap = polish_model.alignment
    rng = np.random.default_rng(12)
    parts, wants = [], []
    for lx, ly in ((0, 0), (0, 9), (9, 0), (1, 1), (5, 40), (40, 5), (30, 33), (64, 64), (80, 77), (118, 120),
                   (170, 160), (230, 228)):
        sx, sy = _rle(rng, lx), _rle(rng, ly)
        strand = int(rng.integers(0, 2))
        rl, rr = bool(rng.integers(0, 2)), bool(rng.integers(0, 2))
        parts.append(Jobs.single(sx, sy, np.zeros((0, 3)), strand, rl, rr))
        m = MpoModel.from_state_model(polish_model.forward if strand else polish_model.reverse)
        wants.append(exact_oracle.forward_probability(m, sx, sy, np.zeros((0, 3)), ap.diagonal_expansion, False,
                                                      rl, rr))
    got = forward_batch(engine, gmodel, ap, Jobs.concat(parts))
    assert got[0] == 0.0
    for g, w in zip(got, wants):
        _ll_close(g, w)


def test_forward_matches_reference_within_logadd(engine, gmodel, polish_model, ref_oracle):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "model_np.npz"))
    hf = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    ap = polish_model.alignment
    jobs = synth.config_small(seed=13, n_reads=2).jobs()
    jobs = Jobs(jobs.x_symbols, jobs.x_begin, jobs.x_end, jobs.y_symbols, jobs.y_offsets, jobs.anchors,
                jobs.anchor_offsets, np.ones(jobs.n_jobs, np.uint8))
    got = forward_batch(engine, gmodel, ap, jobs)
    for j in range(jobs.n_jobs):
        sx, sy, a = _job(jobs, j)
        want = ref_oracle.forward_probability(hf, sx, sy, a, ap)
        assert abs(got[j] - want) <= 2e-3 * abs(want)
    ref_oracle.free_model(hf)


def _oracle_expectations(exact_oracle, polish_model, jobs):
    """Summed FP64 expected counts per strand model, and per-job ln P."""
    ap = polish_model.alignment
    acc = {k: np.zeros((2,) + s) for k, s in (("transitions", (9,)), ("match", (25,)), ("gap_x", (5,)),
                                              ("gap_y", (5,)), ("start", (3,)), ("end", (3,)))}
    rep = np.zeros(4 * 51 * 51)
    lls = []
    for j in range(jobs.n_jobs):
        sx, sy, a = _job(jobs, j)
        md = 0 if jobs.strand[j] else 1
        m = MpoModel.from_state_model(polish_model.forward if md == 0 else polish_model.reverse)
        rl = bool(jobs.ragged_left[j]) if jobs.ragged_left is not None else False
        rr = bool(jobs.ragged_right[j]) if jobs.ragged_right is not None else False
        lp, ex = exact_oracle.expectations(m, sx, sy, a, ap.diagonal_expansion, True, rl, rr)
        for k in acc:
            acc[k][md] += ex[k]
        rep += ex["repeat"]
        lls.append(lp)
    # transitions: the oracle counts exp(f + t + e + b - P) directly
    return acc, rep, np.array(lls)


def _counts_close(got, want):
    got, want = np.asarray(got, float), np.asarray(want, float)
    tol = np.maximum(1e-4, 1e-4 * np.abs(want))
    bad = np.abs(got - want) > tol
    assert not bad.any(), (got[bad][:5], want[bad][:5])


def test_expectations_match_fp64_oracle(engine, gmodel, polish_model, exact_oracle):
    jobs = synth.config_small(seed=15, n_reads=4).jobs()
    rl = np.array([0, 1, 0, 0], np.uint8)
    rr = np.array([0, 0, 1, 0], np.uint8)
    jobs = Jobs(jobs.x_symbols, jobs.x_begin, jobs.x_end, jobs.y_symbols, jobs.y_offsets, jobs.anchors,
                jobs.anchor_offsets, jobs.strand, rl, rr)
    ex = expectations_batch(engine, gmodel, polish_model.alignment, jobs)
    acc, rep, lls = _oracle_expectations(exact_oracle, polish_model, jobs)
    for j in range(jobs.n_jobs):
        _ll_close(ex.job_log_likelihood[j], lls[j])
    _ll_close(ex.log_likelihood, lls.sum())
    for md in range(2):
        _counts_close(ex.transitions[md].reshape(-1), acc["transitions"][md])
        _counts_close(ex.match[md].reshape(-1), acc["match"][md])
        _counts_close(ex.gap_x[md], acc["gap_x"][md])
        _counts_close(ex.gap_y[md], acc["gap_y"][md])
        _counts_close(ex.start[md], acc["start"][md])
        _counts_close(ex.end[md], acc["end"][md])
    # one run-length table serves both strands (rows chosen by strand)
    assert np.all(ex.repeat[1] == 0.0)
    _counts_close(ex.repeat[0].reshape(-1), rep)


def test_expectations_against_finite_differences(engine, gmodel, polish_model, exact_oracle):
    """Central differences (h = 1e-3) of the FP64 ln P against the GPU's expected counts."""
    ap = polish_model.alignment
    jobs = synth.config_small(seed=17, n_reads=1, template_len=500).jobs()
    ex = expectations_batch(engine, gmodel, ap, jobs)
    sx, sy, a = _job(jobs, 0)
    md = 0 if jobs.strand[0] else 1
    m = MpoModel.from_state_model(polish_model.forward if md == 0 else polish_model.reverse)
    e = ap.diagonal_expansion

    def fd(field, k, scale=1.0, h=1e-3):
        arr = getattr(m, field)
        v0 = arr[k]
        arr[k] = v0 + h / scale
        up = exact_oracle.forward_probability(m, sx, sy, a, e, True)
        arr[k] = v0 - h / scale
        dn = exact_oracle.forward_probability(m, sx, sy, a, e, True)
        arr[k] = v0
        return (up - dn) / (2 * h)

    def close(g, w):
        assert abs(g - w) <= max(2e-4, 2e-4 * abs(w)), (g, w)

    for k in range(9):
        if np.isfinite(m.trans[k]):
            close(ex.transitions[md].reshape(-1)[k], fd("trans", k))
    for k in (0, 5, 10, 15, 1, 4):
        close(ex.match[md].reshape(-1)[k], fd("match", k))
    for k in range(4):
        close(ex.gap_x[md][k], fd("gapX", k))
        close(ex.gap_y[md][k], fd("gapY", k))
    for k in range(3):
        close(ex.end[md][k], fd("end", k))
    top = np.argsort(ex.repeat[0].reshape(-1))[::-1][:4]
    for r in top:
        close(ex.repeat[0].reshape(-1)[r], _fd_rep(exact_oracle, m, sx, sy, a, e, r))


def _fd_rep(exact_oracle, m, sx, sy, a, e, r, h=1e-3):
    tab = m._keep
    v0 = tab[r]
    tab[r] = v0 + h / m.repeatScale
    up = exact_oracle.forward_probability(m, sx, sy, a, e, True)
    tab[r] = v0 - h / m.repeatScale
    dn = exact_oracle.forward_probability(m, sx, sy, a, e, True)
    tab[r] = v0
    return (up - dn) / (2 * h)


def test_expected_transitions_match_reference(engine, gmodel, polish_model, ref_oracle):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "model_np.npz"))
    ap = polish_model.alignment
    jobs = synth.config_small(seed=19, n_reads=2).jobs()
    jobs = Jobs(jobs.x_symbols, jobs.x_begin, jobs.x_end, jobs.y_symbols, jobs.y_offsets, jobs.anchors,
                jobs.anchor_offsets, np.ones(jobs.n_jobs, np.uint8))
    hf = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    want = np.zeros(9)
    for j in range(jobs.n_jobs):
        sx, sy, a = _job(jobs, j)
        t, _ = ref_oracle.expectations(hf, int(z["hmm_type"]), sx, sy, a, ap)
        want += t
    ref_oracle.free_model(hf)
    got = expectations_batch(engine, gmodel, ap, jobs).transitions[0].reshape(-1)
    np.testing.assert_allclose(got, want, rtol=2e-3, atol=1e-6)
