"""Generates tests/golden/polish_110kb.npz: the reference's own shipped polishing loop on one chunk
at genome scale, for the GPU polish-identity test (tests/test_gpu_scale.py).

The chunk is the one of make_consensus_golden.py (110 kb homopolymer-enriched truth, draft with 1%
homopolymer-biased indels, 50x log-normal reads, anchors of band half-width 64), here with seeded
nanopore-like base qualities (PolishWorkload.qualities, seed 47) so that the bubble graph's
quality filter takes part. The reference's impl/polisher.c and impl/bubbleGraph.c, compiled
unmodified with its aligner (oracle/_ref/libref_poa.so), run poa_realignAll with the shipped
loop parameters (params/allParams.np.json: no consensus iterations, one polish iteration,
impl/polisher.c:2109-2129) and then the Bayesian run-length estimate (marginPolish.c:554-560);
the fixture holds the polished chunk, the bubble count and a digest of the inputs.

Usage (where the reference build exists; takes several minutes on one core):
    python tests/golden/make_polish_golden.py
"""
import hashlib
import importlib.util
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from marginpolish_b200 import PolishParams, params  # noqa: E402
from oracle.bindings import RefPoaOracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "polish_110kb.npz")
QUAL_SEED = 47


def chunk_workload():
    """The chunk and its qualities (shared with the test, which regenerates them)."""
    spec = importlib.util.spec_from_file_location("mcg", os.path.join(HERE, "make_consensus_golden.py"))
    mcg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mcg)
    wl = mcg.chunk_workload()
    return wl, wl.qualities(QUAL_SEED), mcg.digest


def digest(wl, quals, base_digest) -> str:
    h = hashlib.sha256(base_digest(wl).encode())
    for q in quals[0]:
        h.update(np.asarray(q, np.uint8).tobytes())
    return h.hexdigest()


def main() -> None:
    pm = params.polish_model_from_npz(os.path.join(HERE, "model_np.npz"))
    z = np.load(os.path.join(HERE, "model_np.npz"))
    wl, quals, base_digest = chunk_workload()
    ref = RefPoaOracle()
    hf = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    pp = PolishParams.shipped()
    params_h = ref.params(hf, hr, pm.alignment, max_iterations=pp.max_iterations)
    ref.set_polish(params_h, pp)
    reads_h = ref.reads(wl.reads[0], wl.strands[0])
    ref.set_qualities(reads_h, quals[0])
    anchors_h = ref.anchors(wl.anchors[0])
    t = time.perf_counter()
    poa = ref.realign_all(reads_h, anchors_h, wl.drafts[0], params_h)
    ref.estimate_repeat_counts(poa, reads_h, params_h)
    seconds = time.perf_counter() - t
    chars, counts = ref.reference(poa)
    np.savez_compressed(OUT, chars=np.frombuffer(chars, np.uint8), counts=counts.astype(np.uint16),
                        digest=np.array(digest(wl, quals, base_digest)), reads=np.int64(len(wl.reads[0])),
                        draft_runs=np.int64(len(wl.drafts[0])), reference_seconds=np.float64(seconds))
    print(f"wrote {OUT}: {len(chars)} runs (draft {len(wl.drafts[0])}) from {len(wl.reads[0])} reads in {seconds:.0f} s")
    ref.free_poa(poa)
    ref.free_anchors(anchors_h)
    ref.free_reads(reads_h)
    ref.free_params(params_h)
    ref.free_model(hf)
    ref.free_model(hr)


if __name__ == "__main__":
    main()
