"""Generates tests/golden/ecoli_windows.npz: real nanopore reads and the reference's own polishing
loop on them, for the GPU real-data test (tests/test_gpu_polish.py).

The inputs are the reference's polishing examples (tests/data/polishTestExamples/
20_random_100bp_windows_directional_ecoli_guppy in the MarginPolish tree): 20 windows of
E. coli, each with Guppy-called nanopore reads marked F / R for their strand, the first read
serving as the draft, and the true 100 bp reference. The reference's test
(tests/polisherTest.c:550-600, :736-819) polishes each window with poa_realignAll without
anchors, at most 100 consensus iterations, reference base penalty 0.6 and three polish
iterations, then estimates the run lengths; this script runs that loop with the reference's own
impl/polisher.c and impl/bubbleGraph.c (oracle/_ref/libref_poa.so) in run-length mode and
stores the inputs (run-length encoded), the true references and the reference's polished
windows.

Usage (where the reference tree and its build exist; a few seconds):
    python tests/golden/make_ecoli_golden.py [reference tree]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from marginpolish_b200 import PolishParams, params  # noqa: E402
from marginpolish_b200.rle import RleString  # noqa: E402
from marginpolish_b200.synth import rle_encode  # noqa: E402
from oracle.bindings import RefPoaOracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "ecoli_windows.npz")
EXAMPLES = "tests/data/polishTestExamples/20_random_100bp_windows_directional_ecoli_guppy"
WINDOWS = 20


def loop_params() -> PolishParams:
    """The polish test's parameters (tests/polisherTest.c:563-569) on top of the shipped ones."""
    return PolishParams(reference_base_penalty=0.6, min_iterations=0, max_iterations=100, min_polish_iterations=3,
                        max_polish_iterations=3)


def read_fasta(path):
    names, seqs = [], []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith(">"):
                names.append(line[1:])
                seqs.append([])
            elif line:
                seqs[-1].append(line)
    return names, ["".join(s) for s in seqs]


def encode(seq: str) -> RleString:
    return rle_encode(np.frombuffer(seq.encode(), np.uint8))


def flat(strings):
    off = np.zeros(len(strings) + 1, np.int64)
    off[1:] = np.cumsum([len(s) for s in strings])
    chars = np.frombuffer(b"".join(s.chars for s in strings), np.uint8)
    counts = np.concatenate([np.asarray(s.counts, np.uint32) for s in strings]) if strings else np.zeros(0, np.uint32)
    return off, chars, counts


def main() -> None:
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MP_REFERENCE_TREE")
    if not tree or not os.path.isdir(os.path.join(tree, EXAMPLES)):
        sys.exit("usage: make_ecoli_golden.py <reference tree> (or set MP_REFERENCE_TREE)")
    pm = params.polish_model_from_npz(os.path.join(HERE, "model_np.npz"))
    z = np.load(os.path.join(HERE, "model_np.npz"))
    ref = RefPoaOracle()
    hf = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    pp = loop_params()
    params_h = ref.params(hf, hr, pm.alignment, penalty=pp.reference_base_penalty, min_iterations=pp.min_iterations,
                          max_iterations=pp.max_iterations)
    ref.set_polish(params_h, pp)
    drafts, truths, reads, strands, polished = [], [], [], [], []
    for w in range(WINDOWS):
        names, seqs = read_fasta(os.path.join(tree, EXAMPLES, f"{w}.fasta"))
        _, truth = read_fasta(os.path.join(tree, EXAMPLES, f"{w}.ref.fasta"))
        draft = encode(seqs[0])
        rs = [encode(s) for s in seqs[1:]]
        st = [1 if n.endswith("F") else 0 for n in names[1:]]
        reads_h = ref.reads(rs, st)
        poa = ref.realign_all(reads_h, None, draft, params_h)  # no anchors, as the test runs it
        ref.estimate_repeat_counts(poa, reads_h, params_h)
        chars, counts = ref.reference(poa)
        polished.append(RleString(chars, counts.astype(np.uint32)))
        ref.free_poa(poa)
        ref.free_reads(reads_h)
        drafts.append(draft)
        truths.append(encode(truth[0]))
        reads.append(rs)
        strands.append(st)
    d_off, d_chars, d_counts = flat(drafts)
    t_off, t_chars, t_counts = flat(truths)
    p_off, p_chars, p_counts = flat(polished)
    all_reads = [r for lst in reads for r in lst]
    r_off, r_chars, r_counts = flat(all_reads)
    chunk_reads = np.zeros(WINDOWS + 1, np.int64)
    chunk_reads[1:] = np.cumsum([len(lst) for lst in reads])
    np.savez_compressed(OUT, draft_offsets=d_off, draft_chars=d_chars, draft_counts=d_counts.astype(np.uint16),
                        truth_offsets=t_off, truth_chars=t_chars, truth_counts=t_counts.astype(np.uint16),
                        read_offsets=r_off, read_chars=r_chars, read_counts=r_counts.astype(np.uint16),
                        chunk_reads=chunk_reads, strands=np.concatenate([np.asarray(s, np.uint8) for s in strands]),
                        polished_offsets=p_off, polished_chars=p_chars, polished_counts=p_counts.astype(np.uint16))
    changed = sum(int(p.chars != d.chars or not np.array_equal(p.counts, d.counts)) for p, d in zip(polished, drafts))
    print(f"wrote {OUT}: {WINDOWS} windows, {len(all_reads)} reads, {changed} windows changed by the loop")
    ref.free_params(params_h)
    ref.free_model(hf)
    ref.free_model(hr)


if __name__ == "__main__":
    main()
