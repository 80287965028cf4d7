"""Ingest over the library's C ABI (mp_bam_*): a coordinate-sorted BAM file to the chunks of the
polishing loop (bamChunker_construct2, impl/htsIntegration.c:149-273) and each chunk's reads,
qualities, strands and anchors (convertToReadsAndAlignments, :347-661), plus a FASTA reader for
the draft. Host code (the BAM is read and inflated by the library itself; there is no htslib)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import c_char, c_int32, c_int64, c_uint8, c_uint32
from .rle import RleString


@dataclass
class BamParams:
    """The ingest fields of PolishParams; defaults are the shipped params/allParams.np.json."""
    chunk_size: int = 200_000
    chunk_boundary: int = 50
    include_soft_clip: bool = False
    include_secondary: bool = False
    include_supplementary: bool = False
    use_run_length: bool = True
    min_mapq: int = 60
    region: Optional[str] = None   # "contig:start-end", 0-based start, exclusive end

    def struct(self):
        r = self.region.encode() if self.region else None
        return _lib.BamParamsC(int(self.chunk_size), int(self.chunk_boundary), int(self.include_soft_clip),
                               int(self.include_secondary), int(self.include_supplementary), int(self.use_run_length),
                               int(self.min_mapq), r)


@dataclass
class BamChunk:
    contig: str
    boundary_start: int
    start: int
    end: int
    boundary_end: int


@dataclass
class ChunkReads:
    """One chunk's reads as the loop takes them."""
    reads: List[RleString] = field(default_factory=list)
    qualities: List[Optional[np.ndarray]] = field(default_factory=list)  # per run, None without
    strands: List[int] = field(default_factory=list)
    anchors: List[np.ndarray] = field(default_factory=list)  # (n, 3): reference run, read run, 10
    names: List[str] = field(default_factory=list)


class BamFile:
    """An opened BAM file and its chunks (see mp_bam_open)."""

    def __init__(self, path: str, params: Optional[BamParams] = None):
        self.params = params or BamParams()
        self._lib = _lib.load()
        self._p = self.params.struct()
        h = ctypes.c_void_p()
        _lib.check(self._lib.mp_bam_open(path.encode(), ctypes.byref(self._p), ctypes.byref(h)))
        self.handle = h
        n = c_int64(0)
        _lib.check(self._lib.mp_bam_chunk_count(self.handle, ctypes.byref(n)))
        self.chunks: List[BamChunk] = []
        name = (c_char * 4096)()
        b = np.zeros(4, np.int64)
        for i in range(n.value):
            _lib.check(self._lib.mp_bam_chunk(self.handle, i, name, 4096, _lib.ptr(b, c_int64)))
            self.chunks.append(BamChunk(name.value.decode(), *(int(v) for v in b)))

    def convert(self, first: int = 0, n: Optional[int] = None, references: Optional[Sequence[str]] = None,
                max_depth: int = 0, seed: int = 0) -> List[ChunkReads]:
        """convertToReadsAndAlignments for chunks [first, first + n); references[k] is chunk k's
        reference over its bounds (needed for anchors in run-length mode)."""
        n = len(self.chunks) - first if n is None else n
        ro, rc = None, None
        if references is not None:
            raw = [r.encode() for r in references]
            ro = np.zeros(len(raw) + 1, np.int64)
            ro[1:] = np.cumsum([len(r) for r in raw])
            rc = b"".join(raw) or b"\0"
        _lib.check(self._lib.mp_bam_convert(self.handle, first, n, _lib.ptr(ro, c_int64), rc, int(max_depth),
                                            int(seed)))
        out = []
        for k in range(n):
            sz = np.zeros(4, np.int64)
            _lib.check(self._lib.mp_bam_reads_sizes(self.handle, k, _lib.ptr(sz, c_int64)))
            nr, runs, na, nb = (int(v) for v in sz)
            roff = np.zeros(nr + 1, np.int64)
            chars = (c_char * max(runs, 1))()
            counts = np.zeros(max(runs, 1), np.uint32)
            quals = np.zeros(max(runs, 1), np.uint8)
            hasq = np.zeros(max(nr, 1), np.uint8)
            st = np.zeros(max(nr, 1), np.uint8)
            aoff = np.zeros(nr + 1, np.int64)
            anc = np.zeros((max(na, 1), 3), np.int32)
            noff = np.zeros(nr + 1, np.int64)
            names = (c_char * max(nb, 1))()
            _lib.check(self._lib.mp_bam_reads(self.handle, k, _lib.ptr(roff, c_int64), chars,
                                              _lib.ptr(counts, c_uint32), _lib.ptr(quals, c_uint8),
                                              _lib.ptr(hasq, c_uint8), _lib.ptr(st, c_uint8), _lib.ptr(aoff, c_int64),
                                              _lib.ptr(anc, c_int32), _lib.ptr(noff, c_int64), names))
            raw = bytes(chars[:runs])
            rawn = bytes(names[:nb]).decode()
            cr = ChunkReads()
            for i in range(nr):
                a, b = int(roff[i]), int(roff[i + 1])
                cr.reads.append(RleString(raw[a:b], counts[a:b].copy()))
                cr.qualities.append(quals[a:b].copy() if hasq[i] else None)
                cr.strands.append(int(st[i]))
                cr.anchors.append(anc[aoff[i]:aoff[i + 1]].astype(np.int64))
                cr.names.append(rawn[noff[i]:noff[i + 1]])
            out.append(cr)
        return out

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.mp_bam_close(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_fasta(path: str) -> Dict[str, str]:
    """Sequences of a FASTA file by name (the first word of the header)."""
    seqs: Dict[str, List[str]] = {}
    name = None
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith(">"):
                name = line[1:].split()[0] if len(line) > 1 else ""
                seqs[name] = []
            elif name is not None and line:
                seqs[name].append(line)
    return {k: "".join(v) for k, v in seqs.items()}


def chunk_reference(sequences: Dict[str, str], chunk: BamChunk) -> str:
    """The chunk's reference over its bounds, cut at the sequence's end (marginPolish.c:58-66)."""
    s = sequences[chunk.contig]
    return s[chunk.boundary_start:min(len(s), chunk.boundary_end)]
