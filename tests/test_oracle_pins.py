"""Pins of the two CPU oracles against the reference's own known answers and against each other.

Oracle A is the reference's code compiled unmodified; Oracle B is the FP64 restatement. With the
reference's logAdd plugged into Oracle B the two must agree bit for bit (every tuple of every list,
in order); with the exact log-sum Oracle B is the FP64 oracle the GPU is held to."""
import math

import numpy as np
import pytest

from marginpolish_b200 import AlignmentParams, _lib, synth
from oracle.bindings import MpoModel

# tests/pairwiseAlignerTest.c:64-127 -- anchors (1,0),(2,1),(3,3), lX=6, lY=5, expansion 2
BAND_ANCHORS = np.array([[1, 0, 2], [2, 1, 2], [3, 3, 2]])
BAND_EXPECTED = [(0, 0, 0), (1, -1, 1), (2, -2, 2), (3, -1, 3), (4, -2, 4), (5, -1, 3), (6, -2, 4), (7, -3, 3),
                 (8, -2, 2), (9, -1, 3), (10, 0, 2), (11, 1, 1)]

# tests/pairwiseAlignerTest.c:487-556 -- split rectangles
SPLIT_ANCHORS = np.array([[2000, 2000, 0], [4002, 4001, 0], [5000, 5000, 0], [8000, 6000, 0], [9000, 9000, 0],
                          [10000, 14000, 0], [15000, 15000, 0], [16000, 16000, 0]])
SPLIT_EXPECTED = [(0, 0, 3001, 3001), (3002, 3001, 9500, 11001), (9501, 12000, 12001, 14500),
                  (13000, 14501, 18000, 18001), (18001, 23000, 20000, 25000)]


def _mp_band(anchors, lx, ly, e, dynamic):
    import ctypes
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int32).reshape(-1, 3))
    out = np.zeros((lx + ly + 1, 3), dtype=np.int64)
    _lib.check(_lib.load().mp_band(_lib.ptr(a, ctypes.c_int32) if a.size else None, a.shape[0], lx, ly, e,
                                   int(dynamic), _lib.ptr(out, ctypes.c_int64)))
    return out


def _mp_split(anchors, lx, ly, size, rl, rr):
    import ctypes
    a = np.ascontiguousarray(np.asarray(anchors, dtype=np.int32).reshape(-1, 3))
    out = np.zeros((64, 4), dtype=np.int64)
    n = ctypes.c_int64()
    _lib.check(_lib.load().mp_split_points(_lib.ptr(a, ctypes.c_int32) if a.size else None, a.shape[0], lx, ly, size,
                                           int(rl), int(rr), _lib.ptr(out, ctypes.c_int64), 64, n))
    return [tuple(r) for r in out[:n.value]]


def test_band_known_answer(ref_oracle, exact_oracle):
    for band in (ref_oracle.band(BAND_ANCHORS, 6, 5, 2, False), exact_oracle.band(BAND_ANCHORS, 6, 5, 2, False),
                 _mp_band(BAND_ANCHORS, 6, 5, 2, False)):
        assert [tuple(r) for r in band] == BAND_EXPECTED


def test_split_points_known_answer(ref_oracle, exact_oracle):
    size = 2000 * 2000
    lx, ly = 20000, 25000
    for fn in (lambda *a: [tuple(r) for r in ref_oracle.split_points(*a)],
               lambda *a: [tuple(r) for r in exact_oracle.split_points(*a)], _mp_split):
        assert fn(SPLIT_ANCHORS, lx, ly, size, 0, 0) == SPLIT_EXPECTED
        assert fn(np.zeros((0, 3)), 3000, 1000, size, 0, 0) == [(0, 0, 3000, 1000)]
        assert fn(np.zeros((0, 3)), lx, ly, size, 1, 1) == []
        assert fn(np.zeros((0, 3)), lx, ly, size, 1, 0) == [(18000, 23000, lx, ly)]
        assert fn(np.zeros((0, 3)), lx, ly, size, 0, 1) == [(0, 0, 2000, 2000)]
        assert fn(np.zeros((0, 3)), lx, ly, size, 0, 0) == [(0, 0, 2000, 2000), (18000, 23000, lx, ly)]


def test_reference_logadd_accuracy(ref_oracle):
    """tests/pairwiseAlignerTest.c:129-139: exp(logAdd(log i, log j)) within 1e-3 of i + j."""
    rng = np.random.default_rng(0)
    for i, j in rng.random((20000, 2)):
        assert abs(math.exp(ref_oracle.lib.refo_logadd(math.log(i), math.log(j))) - (i + j)) < 1e-3


def test_random_bands_match_reference(ref_oracle, exact_oracle):
    rng = np.random.default_rng(5)
    for _ in range(200):
        lx, ly = int(rng.integers(0, 60)), int(rng.integers(0, 60))
        a, x, y = [], -1, -1
        while True:
            x += int(rng.integers(1, 8))
            y += int(rng.integers(1, 8))
            if x >= lx or y >= ly:
                break
            a.append((x, y, 2 * int(rng.integers(0, 6))))
        a = np.array(a, dtype=np.int64).reshape(-1, 3)
        e = 2 * int(rng.integers(0, 6))
        dyn = bool(rng.random() < 0.5)
        ra = ref_oracle.band(a, lx, ly, e, dyn)
        assert np.array_equal(ra, exact_oracle.band(a, lx, ly, e, dyn))
        assert np.array_equal(ra, _mp_band(a, lx, ly, e, dyn))


def _models(ref_oracle, polish_model):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "model_np.npz"))
    hf = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    return (hf, hr), (MpoModel.from_state_model(polish_model.forward), MpoModel.from_state_model(polish_model.reverse))


def test_restatement_is_bit_exact_with_reference_on_small_workload(ref_oracle, exact_oracle, polish_model):
    (hf, hr), (mf, mr) = _models(ref_oracle, polish_model)
    jobs = synth.config_small(seed=1).jobs()
    la = ref_oracle.logadd_address()
    for j in range(jobs.n_jobs):
        sx = jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]]
        sy = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        s = jobs.strand[j]
        A = ref_oracle.align_with_indels(hf if s else hr, sx, sy, a, polish_model.alignment)
        B = exact_oracle.align_with_indels(mf if s else mr, sx, sy, a, polish_model.alignment, logadd=la)
        for k in range(3):
            assert np.array_equal(A[k], B["pairs"][k]), f"job {j} list {k}"


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_restatement_is_bit_exact_with_reference_on_segments(ref_oracle, exact_oracle, default_model, seed):
    """Random anchors and traceback parameters small enough to force several traceback segments
    (tests/pairwiseAlignerTest.c:418-455 style), ragged ends, default machine, 'N' symbols.

    Jobs that need split rectangles are excluded here: the reference's symbolString_getSubString
    (impl/stateMachine.c:102-110) copies the whole SymbolString and never sets the sub-string's length,
    so each split sub-problem runs over the full lengths and reads past its symbol buffer (undefined
    behaviour). The GPU is held to the restatement's split semantics (the rectangle's own lengths)."""
    rng = np.random.default_rng(seed)
    d = ref_oracle.default_model()
    m = MpoModel.from_state_model(default_model)
    la = ref_oracle.logadd_address()
    for _ in range(25):
        lx = int(rng.integers(0, 150))
        sx = rng.integers(0, 5, size=lx).astype(np.uint16)
        sy = np.array([c if rng.random() > 0.15 else rng.integers(0, 4) for c in sx if rng.random() > 0.08],
                      dtype=np.uint16)
        a, x, y = [], -1, -1
        while True:
            x += int(rng.integers(1, 20))
            y += int(rng.integers(1, 20))
            if x >= sx.size or y >= sy.size:
                break
            a.append((x, y, 2 * int(rng.integers(0, 5))))
        a = np.array(a, dtype=np.int64).reshape(-1, 3)
        tb = int(rng.integers(1, 10))
        p = AlignmentParams(threshold=0.01, traceback_diagonals=tb, min_diags_between_traceback=tb + int(rng.integers(2, 10)),
                            diagonal_expansion=2 * int(rng.integers(0, 10)), dynamic_anchor_expansion=bool(rng.random() < 0.5),
                            split_matrix_bigger_than_this=int(rng.choice([9000000, 300, 900])))
        rl, rr = bool(rng.random() < 0.3), bool(rng.random() < 0.3)
        if len(exact_oracle.split_points(a, sx.size, sy.size, p.split_matrix_bigger_than_this, rl, rr)) != 1 or \
                any(r != (0, 0, sx.size, sy.size) for r in
                    map(tuple, exact_oracle.split_points(a, sx.size, sy.size, p.split_matrix_bigger_than_this, rl, rr))):
            continue
        A = ref_oracle.align_with_indels(d, sx, sy, a, p, rl, rr)
        B = exact_oracle.align_with_indels(m, sx, sy, a, p, rl, rr, logadd=la)
        for k in range(3):
            assert np.array_equal(A[k], B["pairs"][k])
    ref_oracle.free_model(d)


def test_golden_reference_outputs(exact_oracle, polish_model):
    """The committed Oracle-A outputs (tests/golden/oracle_a_small.npz) against the FP64 restatement.
    The reference's logAdd is a piecewise cubic (impl/pairwiseAligner.c:282-299), so its posteriors differ
    from exact FP64 by up to ~2.4e-3 for large posteriors but by < 1e-5 near the 0.01 threshold: the tuple
    sets agree outside +-1e-4 of the threshold and common weights within 3e-3."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_a_small.npz"))
    ms = (MpoModel.from_state_model(polish_model.reverse), MpoModel.from_state_model(polish_model.forward))
    from oracle.compare import dense_table
    for j in range(int(z["n"])):
        o = exact_oracle.align_with_indels(ms[int(z[f"strand{j}"])], z[f"sx{j}"], z[f"sy{j}"], z[f"anchors{j}"],
                                           polish_model.alignment, dense=True)
        table = dense_table(o["dense"])
        for k, name in enumerate(("match", "gapx", "gapy")):
            ref = {(int(x), int(y)): w for w, x, y in z[f"{name}{j}"]}
            ex = {(int(x), int(y)): w for w, x, y in o["pairs"][k]}
            for key in set(ref) ^ set(ex):
                assert abs(table[key][k] - polish_model.alignment.threshold) < 1e-4
            for key in set(ref) & set(ex):
                assert abs(ref[key] - ex[key]) <= 3e-3 * 1e7  # the reference's logAdd: measured max 2.4e-3
