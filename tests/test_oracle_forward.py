"""CPU pins of the FP64 oracle's forward likelihood and expected counts.

* forward likelihood: with the reference's own logAdd the restatement equals the
  reference's computeForwardProbability (impl/pairwiseAligner.c:813-865) bit for bit,
  with and without anchors and with ragged ends;
* expected transitions: the exact FP64 counts agree with the reference's
  getExpectationsUsingAnchors (impl/pairwiseAligner.c:1151-1156) within the error of
  its approximate logAdd (single traceback segment, as for reads < 10000 diagonals);
* every expected count equals the central finite difference of the FP64 log-likelihood
  with respect to the matching log parameter.
"""
import numpy as np
import pytest

from marginpolish_b200 import synth
from oracle.bindings import MpoModel


def _job(jobs, j):
    sx = jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]]
    sy = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
    a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
    return sx, sy, a


def _ref_models(ref_oracle):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "model_np.npz"))
    hf = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    return int(z["hmm_type"]), hf, hr


def _random_pair(rng, lx, ly):
    """Run-length symbols of two random short sequences (bubble-graph sized)."""
    def rle(n):
        b = rng.integers(0, 4, size=n)
        c = rng.integers(1, 6, size=n)
        return ((c << 8) | b).astype(np.uint16)
    return rle(lx), rle(ly)


def test_forward_probability_bit_exact_with_reference(ref_oracle, exact_oracle, polish_model):
    hmm_type, hf, hr = _ref_models(ref_oracle)
    ap = polish_model.alignment
    wl = synth.config_small(seed=3, n_reads=3)
    jobs = wl.jobs()
    for j in range(jobs.n_jobs):
        sx, sy, a = _job(jobs, j)
        fwd = bool(jobs.strand[j])
        m = MpoModel.from_state_model(polish_model.forward if fwd else polish_model.reverse)
        for rl, rr in ((False, False), (True, False), (False, True)):
            want = ref_oracle.forward_probability(hf if fwd else hr, sx, sy, a, ap, rl, rr)
            got = exact_oracle.forward_probability(m, sx, sy, a, ap.diagonal_expansion, False, rl, rr,
                                                   logadd=ref_oracle.logadd_address())
            assert got == want
    rng = np.random.default_rng(7)
    m = MpoModel.from_state_model(polish_model.forward)
    for lx, ly in ((0, 0), (0, 5), (7, 0), (1, 1), (12, 30), (60, 55), (100, 97)):
        sx, sy = _random_pair(rng, lx, ly)
        for rl, rr in ((False, False), (True, True)):
            want = ref_oracle.forward_probability(hf, sx, sy, np.zeros((0, 3)), ap, rl, rr)
            got = exact_oracle.forward_probability(m, sx, sy, np.zeros((0, 3)), ap.diagonal_expansion, False, rl, rr,
                                                   logadd=ref_oracle.logadd_address())
            assert got == want, (lx, ly, rl, rr)
            exact = exact_oracle.forward_probability(m, sx, sy, np.zeros((0, 3)), ap.diagonal_expansion, False,
                                                     rl, rr)
            assert abs(exact - want) <= 2e-3 * max(1.0, abs(want))
    ref_oracle.free_model(hf)
    ref_oracle.free_model(hr)


def test_expected_transitions_match_reference(ref_oracle, exact_oracle, polish_model):
    hmm_type, hf, hr = _ref_models(ref_oracle)
    ap = polish_model.alignment
    jobs = synth.config_small(seed=5, n_reads=2).jobs()
    for j in range(jobs.n_jobs):
        sx, sy, a = _job(jobs, j)
        fwd = bool(jobs.strand[j])
        m = MpoModel.from_state_model(polish_model.forward if fwd else polish_model.reverse)
        lp, ex = exact_oracle.expectations(m, sx, sy, a, ap.diagonal_expansion, True)
        t_ref, _ = ref_oracle.expectations(hf if fwd else hr, hmm_type, sx, sy, a, ap)
        np.testing.assert_allclose(ex["transitions"], t_ref, rtol=2e-3, atol=1e-6)
        # each emitted symbol of x is matched or deleted, each of y matched or inserted
        assert abs(ex["match"].sum() + ex["gap_x"].sum() - sx.size) < 1e-6 * sx.size
        assert abs(ex["match"].sum() + ex["gap_y"].sum() - sy.size) < 1e-6 * sy.size
        assert abs(ex["repeat"].sum() - ex["match"].sum()) < 1e-6 * sx.size
        assert abs(ex["start"].sum() - 1.0) < 1e-9 and abs(ex["end"].sum() - 1.0) < 1e-9
    ref_oracle.free_model(hf)
    ref_oracle.free_model(hr)


def _fd(exact_oracle, m, sx, sy, a, e, field, index, h=1e-3, scale=1.0):
    arr = getattr(m, field)
    v0 = arr[index]
    arr[index] = v0 + h / scale
    lp = exact_oracle.forward_probability(m, sx, sy, a, e, True)
    arr[index] = v0 - h / scale
    lm = exact_oracle.forward_probability(m, sx, sy, a, e, True)
    arr[index] = v0
    return (lp - lm) / (2 * h)


def test_expected_counts_are_the_gradient(exact_oracle, polish_model):
    """d lnP / d ln(theta) by central differences (h = 1e-3, FP64) = the expected counts."""
    ap = polish_model.alignment
    wl = synth.config_small(seed=9, n_reads=1, template_len=400)
    jobs = wl.jobs()
    sx, sy, a = _job(jobs, 0)
    sm = polish_model.forward if jobs.strand[0] else polish_model.reverse
    m = MpoModel.from_state_model(sm)
    e = ap.diagonal_expansion
    lp, ex = exact_oracle.expectations(m, sx, sy, a, e, True)
    assert lp == pytest.approx(exact_oracle.forward_probability(m, sx, sy, a, e, True), abs=1e-9)
    for k in range(9):
        if np.isfinite(m.trans[k]):
            assert _fd(exact_oracle, m, sx, sy, a, e, "trans", k) == pytest.approx(ex["transitions"][k], rel=1e-5,
                                                                                   abs=1e-6)
    for k in (0, 6, 12, 18, 1, 7):
        assert _fd(exact_oracle, m, sx, sy, a, e, "match", k) == pytest.approx(ex["match"][k], rel=1e-5, abs=1e-6)
    for k in range(4):
        assert _fd(exact_oracle, m, sx, sy, a, e, "gapX", k) == pytest.approx(ex["gap_x"][k], rel=1e-5, abs=1e-6)
        assert _fd(exact_oracle, m, sx, sy, a, e, "gapY", k) == pytest.approx(ex["gap_y"][k], rel=1e-5, abs=1e-6)
    assert _fd(exact_oracle, m, sx, sy, a, e, "start", 0) == pytest.approx(ex["start"][0], rel=1e-5, abs=1e-6)
    for k in range(3):
        assert _fd(exact_oracle, m, sx, sy, a, e, "end", k) == pytest.approx(ex["end"][k], rel=1e-5, abs=1e-6)
    # the most used run-length entries: d/d ln R = d/d (scale * log10 R)
    tab = m._keep
    top = np.argsort(ex["repeat"])[::-1][:3]
    for r in top:
        v0 = tab[r]
        h = 1e-3
        tab[r] = v0 + h / m.repeatScale
        up = exact_oracle.forward_probability(m, sx, sy, a, e, True)
        tab[r] = v0 - h / m.repeatScale
        dn = exact_oracle.forward_probability(m, sx, sy, a, e, True)
        tab[r] = v0
        assert (up - dn) / (2 * h) == pytest.approx(ex["repeat"][r], rel=1e-5, abs=1e-6)
