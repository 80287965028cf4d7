"""Chunk stitching on the GPU (mp_merge_contig: mergeContigChunks, impl/chunker.c:50-112, with
removeOverlap, impl/polisher.c:1937-2006) against the reference's own removeOverlap.

Polished chunks of a contig overlap by twice the chunk boundary (100 characters shipped); at
every boundary both are cut at the first heaviest match pair of a ragged, anchor-free alignment
with the code-default nucleotide machine. Over an overlap of near-identical sequence the weights
form a plateau, so the GPU computes them in the reference's arithmetic
(mp_match_pairs_reference, checked tuple by tuple against the reference's getAlignedPairs). The
cuts are then compared with the reference's removeOverlap boundary by boundary, and the merged
contig with the reference's merge walk (restated here over the reference's removeOverlap),
including a missing chunk (a spacer of Ns), a chunk too short to keep the previous window, and a
chunk that shares nothing with its neighbour.
"""
import os

import numpy as np
import pytest

from marginpolish_b200 import Jobs, Model, match_pairs_reference, merge_contig, merge_contig_threaded, params

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def ref_poa():
    from oracle.bindings import RefPoaOracle, available_reference_poa
    if not available_reference_poa():
        pytest.skip("reference POA build (oracle/_ref/libref_poa.so) not present")
    return RefPoaOracle()


@pytest.fixture(scope="module")
def stitch_env(engine, polish_model, ref_poa):
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    hf = ref_poa.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref_poa.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    params_h = ref_poa.params(hf, hr, polish_model.alignment, max_iterations=0)
    default = params.code_default_state_model()
    gm = Model(engine, default, default)
    yield gm, params_h
    gm.close()
    ref_poa.free_params(params_h)
    ref_poa.free_model(hf)
    ref_poa.free_model(hr)


def test_reference_arithmetic_pairs_equal_the_reference(engine, stitch_env, polish_model, ref_oracle):
    """mp_match_pairs_reference against the reference's own getAlignedPairs (Oracle A) with its
    code-default nucleotide machine: every tuple, weight and order, for stitching-sized windows of
    related and unrelated sequence, ragged and not."""
    gm, _ = stitch_env
    rng = np.random.default_rng(17)
    d = ref_oracle.default_model()
    parts, want = [], []
    for k in range(12):
        n = int(rng.integers(1, 120))
        sx = rng.integers(0, 5 if k % 4 == 3 else 4, size=n).astype(np.uint16)
        sy = sx.copy() if k % 3 else rng.integers(0, 4, size=int(rng.integers(1, 120))).astype(np.uint16)
        flip = rng.random(sy.size) < 0.05
        sy[flip] = rng.integers(0, 4, size=int(flip.sum()))
        rl, rr = bool(k % 2), bool((k // 2) % 2)
        parts.append(Jobs.single(sx, sy, np.zeros((0, 3)), 1, rl, rr))
        want.append(ref_oracle.align_with_indels(d, sx, sy, np.zeros((0, 3)), polish_model.alignment, rl, rr)[0])
    got = match_pairs_reference(engine, gm, polish_model.alignment, Jobs.concat(parts))
    for g, w in zip(got, want):
        assert np.array_equal(g, np.asarray(w, np.int64).reshape(-1, 3))
    assert sum(g.shape[0] for g in got) > 300
    ref_oracle.free_model(d)


def _mutate(rng, s: str, rate: float) -> str:
    out = []
    for ch in s:
        r = rng.random()
        if r < rate / 3:
            continue  # deletion
        if r < 2 * rate / 3:
            out.append("ACGT"[rng.integers(4)])  # substitution
        else:
            out.append(ch)
        if rng.random() < rate / 3:
            out.append("ACGT"[rng.integers(4)])  # insertion
    return "".join(out)


def _contig(seed, n_chunks=8, chunk=400, boundary=50, rate=0.004):
    """Polished chunks of one synthetic contig: each covers its 400 bases plus the boundary on
    both sides, with independent residual errors (so overlaps differ a little)."""
    rng = np.random.default_rng(seed)
    truth = "".join("ACGT"[i] for i in rng.integers(0, 4, size=n_chunks * chunk + 2 * boundary))
    chunks = []
    for c in range(n_chunks):
        a = max(0, c * chunk - boundary)
        b = min(len(truth), (c + 1) * chunk + boundary)
        chunks.append(_mutate(rng, truth[a:b], rate))
    return truth, chunks


def _reference_merge(ref_poa, params_h, chunks, overlap, spacer):
    """mergeContigChunks' walk (impl/chunker.c:56-108) over the reference's removeOverlap."""
    pieces, crops = [], []
    for cur in chunks:
        if pieces:
            prev = pieces[-1]
            w, pend, sstart = ref_poa.remove_overlap(prev, cur, overlap, params_h)
            crops.append((w, pend, sstart))
            if w > 0:
                pieces[-1] = prev[:pend]
                cur = cur[sstart:]
            elif len(cur) == 0:
                cur = spacer
            elif overlap != 0:
                pieces.append("N" * 10)
        pieces.append(cur)
    return "".join(pieces), crops


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_merged_contig_matches_reference(engine, stitch_env, polish_model, ref_poa, seed):
    gm, params_h = stitch_env
    overlap, spacer = 100, "N" * 150
    truth, chunks = _contig(seed)
    if seed == 2:
        chunks[3] = ""                     # a missing chunk: its neighbours meet a spacer
        chunks[5] = chunks[5][:70]         # shorter than the window: the next boundary is re-aligned
    if seed == 3:
        rng = np.random.default_rng(9)
        chunks[4] = "".join("ACGT"[i] for i in rng.integers(0, 4, size=300))  # unrelated to its neighbours
    got, report = merge_contig(engine, gm, polish_model.alignment, chunks, overlap, len(spacer))
    want, crops = _reference_merge(ref_poa, params_h, chunks, overlap, spacer)
    same_crop = sum(int((w > 0) == (report[c + 1, 0] > 0) and (w == 0 or report[c + 1, 1] == sstart))
                    for c, (w, _, sstart) in enumerate(crops))
    weight_err = max((abs(int(report[c + 1, 0]) - w) for c, (w, _, _) in enumerate(crops)), default=0)
    print(f"seed {seed}: {len(chunks)} chunks, merged {len(got)} vs reference {len(want)} characters, "
          f"{same_crop}/{len(crops)} crops where the reference cuts, max weight difference {weight_err}")
    assert got == want
    assert same_crop == len(crops)
    assert weight_err <= 1  # CUDA's exp may differ from the host library's in the last place
    if seed == 1:  # the chunks cover the truth up to its last boundary, up to residual indels
        assert abs(len(got) - (len(truth) - 50)) < 20


def test_overlap_zero_and_single_chunk(engine, stitch_env, polish_model):
    gm, _ = stitch_env
    _, chunks = _contig(4, n_chunks=3)
    got, report = merge_contig(engine, gm, polish_model.alignment, chunks, 0, 50)
    assert got == "".join(chunks) and report[:, 2].tolist() == [0, 0, 0]
    got, _ = merge_contig(engine, gm, polish_model.alignment, chunks[:1], 100)
    assert got == chunks[0]


KA_CHUNKS = ["AAAAAAAACC", "AACCCCCCCCGG", "CCGGGGGGGGTT", "GGTTTTTTTT"]
KA_THREADED = ["AAAAAAAACC", "AACCCCCCCCGG", "CCGGGGGGGGTT"] + \
    ["GGTTTTTTTTAA", "TTAAAAAAAACC", "AACCCCCCCCGG", "CCGGGGGGGGTT"] * 3 + ["GGTTTTTTTT"]
KA_TRUTH = "AAAAAAAACCCCCCCCGGGGGGGGTTTTTTTT"


@pytest.fixture(scope="module")
def default_model(engine):
    default = params.code_default_state_model()
    gm = Model(engine, default, default)
    yield gm
    gm.close()


def test_merge_known_answers(engine, default_model, polish_model):
    """test_mergeContigChunks and test_mergeContigChunksThreaded (tests/chunkingTest.c:907-960):
    overlap 4, spacer "NNNNNN", with 1 to 8 merge groups."""
    gm = default_model
    got, report = merge_contig(engine, gm, polish_model.alignment, KA_CHUNKS, 4, 6)
    assert got == KA_TRUTH
    assert (report[1:, 0] > 0).all()
    assert len(KA_THREADED) == 16
    for groups in range(1, 9):
        assert merge_contig_threaded(engine, gm, polish_model.alignment, KA_THREADED, 4, groups, 6) == KA_TRUTH * 4
