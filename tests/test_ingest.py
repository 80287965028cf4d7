"""Ingest (mp_bam_*: bamChunker_construct2 and convertToReadsAndAlignments,
impl/htsIntegration.c:149-273, :347-661) against the known answers of the reference's own
chunking test (tests/chunkingTest.c), on its alignments written as a BAM file
(tests/golden/make_ingest_golden.py). Host code only: runs without a GPU.

The reference test runs with run-length encoding off and no reference sequence; the run-length
cases below check the run-length forms (rleString_rleQualities, runLengthEncodeAlignment,
impl/polisher.c:1692-1750) against the library's own RleString / rle_anchors."""
import json
import os

import numpy as np
import pytest

from marginpolish_b200 import _lib
from marginpolish_b200.ingest import BamFile, BamParams, chunk_reference, read_fasta
from marginpolish_b200.rle import RleString, rle_anchors

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
BAM = os.path.join(GOLDEN, "chunking_test.bam")


def _open(size, boundary, soft_clip=False, region=None, **kw):
    return BamFile(BAM, BamParams(chunk_size=size, chunk_boundary=boundary, include_soft_clip=soft_clip,
                                  use_run_length=False, min_mapq=0, region=region, **kw))


def _bounds(c):
    return (c.contig, c.boundary_start, c.boundary_end)


def test_region_chunker():
    """test_getRegionChunker (tests/chunkingTest.c:23-53)."""
    b = _open(0, 0, region="contig_1:100000-110000")
    assert [_bounds(c) for c in b.chunks] == [("contig_1", 100000, 100008)]
    b = _open(0, 0, region="contig_1:0-3000000")
    assert [_bounds(c) for c in b.chunks] == [("contig_1", 100000, 2100008)]
    b = _open(100000, 0, region="contig_1:100000-300000")
    assert [_bounds(c) for c in b.chunks] == [("contig_1", 100000, 200000), ("contig_1", 200000, 210020)]


def test_chunks_by_contig_and_by_100kb():
    """test_getChunksByChrom and test_getChunksBy100kb (:55-70)."""
    assert len(_open(0, 0).chunks) == 2
    assert len(_open(100000, 0).chunks) == 22


def test_quality_scores():
    """test_getQualityScores (:72-142): the nine reads of contig_2, with and without qualities."""
    b = _open(10000, 0)
    ks = [k for k, c in enumerate(b.chunks) if c.contig == "contig_2"]
    assert ks
    for k in ks:
        cr = b.convert(k, 1)[0]
        assert len(cr.reads) == 9
        j = np.arange(8)
        want = [15 + j, 22 - j, 32 + j, np.zeros(8), np.full(8, 9)]
        for i in range(9):
            if i < 5:
                assert cr.qualities[i] is not None and np.array_equal(cr.qualities[i][:8], want[i])
            else:
                assert cr.qualities[i] is None


@pytest.mark.parametrize("boundary,counts", [(4, [3, 5, 5, 5, 3]), (0, [2, 3, 3, 3, 2])])
def test_chunk_boundaries(boundary, counts):
    """test_getChunksWithBoundary / WithoutBoundary (:144-235): a read is in a chunk when its
    alignment overlaps the chunk's bounds (start inclusive, end exclusive)."""
    b = _open(8, boundary)
    ks = [k for k, c in enumerate(b.chunks) if c.contig == "contig_2"]
    got = [len(b.convert(k, 1)[0].reads) for k in ks]
    assert got == counts


@pytest.mark.parametrize("soft_clip", [False, True])
def test_clipped_reads(soft_clip):
    """test_getReadsWith{,out}SoftClipping (:237-318): soft and hard clips, with insertions and
    deletions, leave 8, 4 or 6 aligned pairs."""
    b = _open(100000, 0, soft_clip)
    ks = [k for k, c in enumerate(b.chunks) if _bounds(c) == ("contig_1", 200000, 300000)]
    assert len(ks) == 1
    cr = b.convert(ks[0], 1)[0]
    assert len(cr.reads) == 10
    want = {3: 4, 5: 6}
    assert [len(a) for a in cr.anchors] == [want.get(i, 8) for i in range(10)]


CASES = {
    "test_readAlignmentsWithoutSoftclippingChunkStart": (1000, False, 400000, 401000),
    "test_readAlignmentsWithSoftclippingChunkStart": (1000, True, 400000, 401000),
    "test_readAlignmentsWithoutSoftclippingChunkEnd": (20, False, 410000, 410020),
    "test_readAlignmentsWithSoftclippingChunkEnd": (20, True, 410000, 410020),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_read_alignments_at_chunk_ends(case):
    """test_readAlignments{With,Without}SoftclippingChunk{Start,End} (:330-900): reads cut at
    the chunk's start and end, each read's sequence and every aligned pair (reference, read)."""
    with open(os.path.join(GOLDEN, "chunking_known_answers.json")) as f:
        ka = json.load(f)[case]
    size, soft, start, end = CASES[case]
    b = _open(size, 0, soft)
    ks = [k for k, c in enumerate(b.chunks) if _bounds(c) == ("contig_1", start, end)]
    assert len(ks) == 1
    cr = b.convert(ks[0], 1)[0]
    assert len(cr.reads) == ka["reads"]
    assert ka["expected"]
    for idx, e in ka["expected"].items():
        i = int(idx)
        assert cr.reads[i].expand() == e["sequence"], (case, i)
        got = cr.anchors[i][:, :2].tolist()
        assert got == e["pairs"], (case, i)
        assert (cr.anchors[i][:, 2] == 10).all() if len(cr.anchors[i]) else True


def test_run_length_forms():
    """With run lengths on, every read is its own RleString, its qualities are one per run (the
    maximum over the run, rleString_rleQualities) and its anchors are runLengthEncodeAlignment's
    of the expanded pairs against the chunk's reference."""
    plain = _open(1000, 0, True)
    rle = BamFile(BAM, BamParams(chunk_size=1000, chunk_boundary=0, include_soft_clip=True, use_run_length=True,
                                 min_mapq=0))
    assert [_bounds(c) for c in plain.chunks] == [_bounds(c) for c in rle.chunks]
    k = [k for k, c in enumerate(rle.chunks) if _bounds(c) == ("contig_1", 400000, 401000)][0]
    c = rle.chunks[k]
    rng = np.random.default_rng(5)
    ref = "".join("ACGT"[i] for i in rng.integers(0, 4, size=c.boundary_end - c.boundary_start))
    p = plain.convert(k, 1)[0]
    r = rle.convert(k, 1, references=[ref])[0]
    assert len(p.reads) == len(r.reads) > 0
    ref_rle = RleString.from_string(ref)
    for i in range(len(p.reads)):
        s = p.reads[i].expand()
        want = RleString.from_string(s)
        assert r.reads[i].chars == want.chars and np.array_equal(r.reads[i].counts, want.counts)
        if p.qualities[i] is not None:
            q = p.qualities[i]
            ends = np.cumsum(want.counts)
            starts = ends - want.counts
            assert np.array_equal(r.qualities[i], [q[a:e].max() for a, e in zip(starts, ends)])
        else:
            assert r.qualities[i] is None
        assert np.array_equal(r.anchors[i], rle_anchors(p.anchors[i], ref_rle, want))
    # without the reference there are no anchors in run-length mode
    r0 = rle.convert(k, 1)[0]
    assert all(len(a) == 0 for a in r0.anchors)


def test_filters_and_errors(tmp_path):
    """Reads below the mapping-quality threshold are dropped; bad inputs raise."""
    every = _open(100000, 0)
    k = [k for k, c in enumerate(every.chunks) if _bounds(c) == ("contig_1", 200000, 300000)][0]
    n = len(every.convert(k, 1)[0].reads)
    strict = BamFile(BAM, BamParams(chunk_size=100000, chunk_boundary=0, use_run_length=False, min_mapq=255))
    assert len(strict.convert(k, 1)[0].reads) < n
    with pytest.raises(_lib.MpError):
        BamFile(str(tmp_path / "missing.bam"))
    junk = tmp_path / "junk.bam"
    junk.write_bytes(b"not a bam file at all")
    with pytest.raises(_lib.MpError):
        BamFile(str(junk))
    assert _open(100, 0, region="no_such_contig:0-10").chunks == []  # as the reference: no chunks
    for bad in ("contig_1", "contig_1:10-5", "contig_1:-1-5", ":0-10"):  # impl/htsIntegration.c:156-163
        with pytest.raises(_lib.MpError):
            _open(100, 0, region=bad)
    with pytest.raises(_lib.MpError):
        every.convert(len(every.chunks), 1)


def test_fasta_reader(tmp_path):
    fa = tmp_path / "draft.fa"
    fa.write_text(">contig_1 polished\nACGT\nAC\n>contig_2\n\nGGG\n")
    seqs = read_fasta(str(fa))
    assert seqs == {"contig_1": "ACGTAC", "contig_2": "GGG"}
    b = _open(0, 0)
    c = b.chunks[0]
    assert chunk_reference({c.contig: "A" * 100}, c) == ""
