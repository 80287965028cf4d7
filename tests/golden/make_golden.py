"""Generates the committed golden fixtures under tests/golden/ (run where the
MarginPolish tree is available; the GPU box only reads the .npz outputs).

* model_np.npz -- the HMM, repeat-count table and banding parameters of the
  reference's params/allParams.np.json ("polish" section), parsed as the
  reference's parser does; plus the code-default machine's lowered tables
  (transitions, emissions, boundaries) probed from the reference's own
  stateMachine3_constructNucleotide through Oracle A.
* oracle_a_small.npz -- the reference's own output (Oracle A:
  getAlignedPairsWithIndelsUsingAnchors) for the first reads of the seeded
  small synthetic workload, with the inputs that produced them.

Usage: python tests/golden/make_golden.py [path/to/reference]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from marginpolish_b200 import params, synth  # noqa: E402
from oracle.bindings import RefOracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main(ref: str) -> None:
    pm = params.load_polish_model(os.path.join(ref, "params", "allParams.np.json"))
    hmm = pm.raw["hmmForwardStrandReadGivenReference"]
    ap = pm.alignment
    ra = RefOracle()
    d = ra.default_model()
    default_trans = ra.transitions(d)
    default_match = np.array([[ra.match_emission(d, x, y) for y in range(5)] for x in range(5)]).reshape(-1)
    default_gap = np.array([ra.gap_emissions(d, c) for c in range(5)])
    default_bound = np.stack([ra.boundary(d, k) for k in range(4)])
    ra.free_model(d)
    np.savez_compressed(
        os.path.join(OUT, "model_np.npz"),
        hmm_type=np.int64(hmm["type"]), transitions=np.asarray(hmm["transitions"], dtype=np.float64),
        emissions=np.asarray(hmm["emissions"], dtype=np.float64), repeat_log10=pm.repeat_log10,
        use_rle=np.int64(pm.use_run_length_encoding), use_repeat_counts=np.int64(pm.use_repeat_counts),
        threshold=np.float64(ap.threshold), min_diags=np.int64(ap.min_diags_between_traceback),
        traceback_diags=np.int64(ap.traceback_diagonals), diagonal_expansion=np.int64(ap.diagonal_expansion),
        constraint_trim=np.int64(ap.constraint_diagonal_trim), split=np.int64(ap.split_matrix_bigger_than_this),
        dynamic=np.int64(ap.dynamic_anchor_expansion), gap_gamma=np.float64(ap.gap_gamma),
        default_transitions=default_trans, default_match=default_match, default_gap=default_gap,
        default_boundary=default_bound)

    # Oracle A outputs on the first reads of the small workload
    wl = synth.config_small(seed=1)
    jobs = wl.jobs()
    hf = ra.model(hmm["type"], hmm["transitions"], hmm["emissions"], False, pm.repeat_log10, 1)
    hr = ra.model(hmm["type"], hmm["transitions"], hmm["emissions"], True, pm.repeat_log10, 0)
    n = 6
    rec = {}
    for j in range(n):
        sx = jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]]
        sy = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        res = ra.align_with_indels(hf if jobs.strand[j] else hr, sx, sy, a, ap)
        rec[f"sx{j}"] = sx
        rec[f"sy{j}"] = sy
        rec[f"anchors{j}"] = a
        rec[f"strand{j}"] = np.int64(jobs.strand[j])
        for k, name in enumerate(("match", "gapx", "gapy")):
            rec[f"{name}{j}"] = res[k].astype(np.int32)
    rec["n"] = np.int64(n)
    np.savez_compressed(os.path.join(OUT, "oracle_a_small.npz"), **rec)
    ra.free_model(hf)
    ra.free_model(hr)
    print("wrote", os.listdir(OUT))


if __name__ == "__main__":
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MP_REFERENCE_TREE")
    if not tree:
        sys.exit("usage: make_golden.py <reference tree> (or set MP_REFERENCE_TREE)")
    main(tree)
