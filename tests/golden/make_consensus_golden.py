"""Generates tests/golden/consensus_110kb.npz: the reference's own polishing loop on one chunk at
genome scale, for the GPU consensus-identity test (tests/test_gpu_scale.py).

The chunk is the first chunk of the seeded 1 Mb polishing configuration: a 110 kb
homopolymer-enriched synthetic truth (100 kb plus 10 kb overlap), a draft with 1%
homopolymer-biased indels, 50x coverage of log-normal reads (median 20 kb, sigma 0.6, at
most 100 kb) with nanopore-like errors, anchors of band half-width 64. The reference's
impl/polisher.c, compiled unmodified with its aligner (oracle/_ref/libref_poa.so), runs
poa_realignAll in consensus mode (up to 5 iterations, impl/polisher.c:2034-2129) and the
Bayesian run-length estimate (:1556-1565); the fixture holds the resulting consensus and a
digest of the inputs, so that the test can tell a changed generator from a changed result.

Usage (where the reference build exists; takes several minutes on one core):
    python tests/golden/make_consensus_golden.py
"""
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from marginpolish_b200 import params, synth  # noqa: E402
from oracle.bindings import RefPoaOracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "consensus_110kb.npz")


def chunk_workload():
    """The chunk (shared with the test, which regenerates it)."""
    return synth.config_polish(seed=47, n_chunks=1, chunk_len=110_000, coverage=50, half_width=64, hp_runs=True,
                               read_lognormal=(20_000, 0.6, 100_000))


def digest(wl) -> str:
    h = hashlib.sha256()
    h.update(wl.drafts[0].chars)
    h.update(np.asarray(wl.drafts[0].counts, np.uint32).tobytes())
    for r, s, a in zip(wl.reads[0], wl.strands[0], wl.anchors[0]):
        h.update(r.chars)
        h.update(np.asarray(r.counts, np.uint32).tobytes())
        h.update(bytes([s]))
        h.update(np.asarray(a, np.int32).tobytes())
    return h.hexdigest()


def main() -> None:
    pm = params.polish_model_from_npz(os.path.join(ROOT, "tests", "golden", "model_np.npz"))
    z = np.load(os.path.join(ROOT, "tests", "golden", "model_np.npz"))
    wl = chunk_workload()
    ref = RefPoaOracle()
    hf = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    params_h = ref.params(hf, hr, pm.alignment, max_iterations=5)
    reads_h = ref.reads(wl.reads[0], wl.strands[0])
    anchors_h = ref.anchors(wl.anchors[0])
    t = time.perf_counter()
    poa = ref.realign_all(reads_h, anchors_h, wl.drafts[0], params_h)
    ref.estimate_repeat_counts(poa, reads_h, params_h)
    seconds = time.perf_counter() - t
    chars, counts = ref.reference(poa)
    np.savez_compressed(OUT, chars=np.frombuffer(chars, np.uint8), counts=counts.astype(np.uint16),
                        digest=np.array(digest(wl)), reads=np.int64(len(wl.reads[0])),
                        draft_runs=np.int64(len(wl.drafts[0])), reference_seconds=np.float64(seconds))
    print(f"wrote {OUT}: {len(chars)} runs from {len(wl.reads[0])} reads in {seconds:.0f} s")
    ref.free_poa(poa)
    ref.free_anchors(anchors_h)
    ref.free_reads(reads_h)
    ref.free_params(params_h)
    ref.free_model(hf)
    ref.free_model(hr)


if __name__ == "__main__":
    main()
