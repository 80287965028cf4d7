"""Host-side interface of the POA loop (impl/polisher.c), mirroring the reference's
operator API over the library's C ABI (mp_poa_set_*):

* ``PoaSet.realign``        -- poa_realign (:656-703) of every chunk (one GPU batch);
* ``PoaSet.realign_pairs``  -- poa_augment (:316-534) with aligned pairs from the caller;
* ``PoaSet.consensus``      -- poa_getConsensus (:1025-1275);
* ``PoaSet.anchor_alignments`` -- poa_getAnchorAlignments (:536-592);
* ``PoaSet.estimate_repeat_counts`` -- poa_estimateRepeatCountsUsingBayesianModel (:1556-1565);
* ``PoaSet.iterate`` / ``iterate_polish`` / ``realign_all`` -- poa_realignIterative in
  consensus or polish mode and poa_realignAll (:2034-2129);
* ``PoaSet.build_bubbles`` / ``score_bubbles`` / ``bubbles`` / ``bubble_consensus`` -- the
  steps of poa_polish (:2008-2031): bubbleGraph_constructFromPoa, the allele scores (one
  GPU launch for all chunks), the allele choice and the new consensus (impl/bubbleGraph.c);
* ``polish`` -- the whole loop for many chunks, returning each chunk's polished draft.

Weights, observations and indels can be read back for every chunk, with the layouts of
the reference's Poa structures (inc/margin.h:592-627).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import c_char, c_double, c_int32, c_int64, c_uint8, c_uint32, c_void_p
from .params import AlignmentParams, PolishModel
from .realign import Engine, Model
from .rle import RleString

c_uint64 = ctypes.c_uint64


@dataclass
class PolishParams:
    """The POA fields of PolishParams (inc/margin.h:534-580). Defaults are the shipped
    params/allParams.np.json values except the iteration counts: these defaults run the
    consensus mode (max_iterations 5) and no polish mode; ``shipped()`` gives the shipped loop
    (no consensus iterations, one polish iteration)."""
    reference_base_penalty: float = 0.5
    compare_repeat_counts: bool = True
    use_run_length: bool = True
    anchor_probs: Sequence[float] = (0.9, 10, 0.95, 4, 0.99, 0)
    min_iterations: int = 0
    max_iterations: int = 5
    # polish mode (poa_polish)
    min_polish_iterations: int = 0
    max_polish_iterations: int = 0
    use_read_alleles: bool = True
    candidate_variant_weight: float = 0.18
    column_anchor_trim: int = 5
    filter_reads_coverage: int = 15
    min_avg_base_quality: float = 10.0
    max_consensus_strings: int = 100

    @classmethod
    def shipped(cls) -> "PolishParams":
        """The loop params/allParams.np.json configures: poa_realignAll with no consensus
        iterations and one polish iteration (impl/polisher.c:2109-2129)."""
        return cls(min_iterations=0, max_iterations=0, min_polish_iterations=1, max_polish_iterations=1)

    def struct(self):
        probs = np.ascontiguousarray(self.anchor_probs, dtype=np.float64)
        p = _lib.PolishParamsC(float(self.reference_base_penalty), 1 if self.compare_repeat_counts else 0,
                               1 if self.use_run_length else 0, _lib.ptr(probs, c_double), probs.size,
                               int(self.min_iterations), int(self.max_iterations), int(self.min_polish_iterations),
                               int(self.max_polish_iterations), 1 if self.use_read_alleles else 0, 0,
                               float(self.candidate_variant_weight), int(self.column_anchor_trim),
                               int(self.filter_reads_coverage), float(self.min_avg_base_quality))
        return p, probs


def _flat_rle(strings: Sequence[RleString]):
    offs = np.zeros(len(strings) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(s) for s in strings])
    chars = b"".join(s.chars for s in strings)
    counts = (np.concatenate([np.asarray(s.counts, dtype=np.uint32) for s in strings])
              if strings else np.zeros(0, np.uint32))
    return offs, chars, np.ascontiguousarray(counts, dtype=np.uint32)


class PoaSet:
    """Chunks (a draft and its reads each) polished together; see mp_poa_set_create. engine
    and model may be None for a set fed with realign_pairs (host-side steps only)."""

    def __init__(self, engine: Engine, model: Model, params: AlignmentParams, polish: PolishParams,
                 drafts: Sequence[RleString], reads: Sequence[Sequence[RleString]], strands: Sequence[Sequence[int]],
                 anchors: Optional[Sequence[Sequence[np.ndarray]]] = None, repeat_log10: Optional[np.ndarray] = None,
                 qualities: Optional[Sequence[Sequence[np.ndarray]]] = None):
        self.engine, self.model = engine, model
        self._lib = engine._lib if engine is not None else _lib.load()
        self.n_chunks = len(drafts)
        flat_reads = [r for lst in reads for r in lst]
        self.reads_per_chunk = [len(lst) for lst in reads]
        ref_off, ref_chars, ref_counts = _flat_rle(list(drafts))
        rd_off, rd_chars, rd_counts = _flat_rle(flat_reads)
        chunk_reads = np.zeros(self.n_chunks + 1, dtype=np.int64)
        chunk_reads[1:] = np.cumsum(self.reads_per_chunk)
        strand = np.ascontiguousarray([int(s) for lst in strands for s in lst], dtype=np.uint8)
        if strand.size != len(flat_reads):
            raise ValueError("one strand per read")
        keep = [ref_off, ref_counts, rd_off, rd_counts, chunk_reads, strand]
        b = _lib.PolishBatch()
        b.n_chunks = self.n_chunks
        b.ref_offsets = _lib.ptr(ref_off, c_int64)
        self._ref_chars = ctypes.create_string_buffer(ref_chars or b"\0", max(len(ref_chars), 1))
        b.ref_chars = ctypes.cast(self._ref_chars, ctypes.POINTER(c_char))
        b.ref_counts = _lib.ptr(ref_counts if ref_counts.size else np.zeros(1, np.uint32), c_uint32)
        b.chunk_reads = _lib.ptr(chunk_reads, c_int64)
        b.read_offsets = _lib.ptr(rd_off, c_int64)
        self._rd_chars = ctypes.create_string_buffer(rd_chars or b"\0", max(len(rd_chars), 1))
        b.read_chars = ctypes.cast(self._rd_chars, ctypes.POINTER(c_char))
        b.read_counts = _lib.ptr(rd_counts if rd_counts.size else np.zeros(1, np.uint32), c_uint32)
        b.strand = _lib.ptr(strand if strand.size else np.zeros(1, np.uint8), c_uint8)
        if anchors is not None:
            flat_a = [np.asarray(a, dtype=np.int32).reshape(-1, 3) for lst in anchors for a in lst]
            a_off = np.zeros(len(flat_a) + 1, dtype=np.int64)
            a_off[1:] = np.cumsum([a.shape[0] for a in flat_a])
            a_all = np.ascontiguousarray(np.concatenate(flat_a) if flat_a else np.zeros((1, 3), np.int32))
            keep += [a_off, a_all]
            b.anchor_offsets = _lib.ptr(a_off, c_int64)
            b.anchors = _lib.ptr(a_all, c_int32)
        if qualities is not None:
            flat_q = [np.asarray(q, dtype=np.uint8) for lst in qualities for q in lst]
            if len(flat_q) != len(flat_reads) or any(q.size != len(r) for q, r in zip(flat_q, flat_reads)):
                raise ValueError("one quality per read run")
            q_all = np.ascontiguousarray(np.concatenate(flat_q) if flat_q and rd_off[-1] else np.zeros(1, np.uint8))
            keep.append(q_all)
            b.read_qualities = _lib.ptr(q_all, c_uint8)
        pp, probs = polish.struct()
        keep.append(probs)
        ps = params.struct()
        rep = None
        if repeat_log10 is not None:
            rep = np.ascontiguousarray(repeat_log10, dtype=np.float64).reshape(-1)
            keep.append(rep)
        self._keep = keep
        h = c_void_p()
        _lib.check(self._lib.mp_poa_set_create(engine.handle if engine is not None else None,
                                               model.handle if model is not None else None, ctypes.byref(ps),
                                               ctypes.byref(pp), ctypes.byref(b), _lib.ptr(rep, c_double),
                                               ctypes.byref(h)))
        self.handle = h

    @classmethod
    def from_polish_model(cls, engine, model, pm: PolishModel, polish: PolishParams, drafts, reads, strands,
                          anchors=None, qualities=None) -> "PoaSet":
        return cls(engine, model, pm.alignment, polish, drafts, reads, strands, anchors,
                   pm.repeat_log10 if polish.use_run_length else None, qualities)

    # ---- the loop's steps ----
    def realign(self) -> None:
        _lib.check(self._lib.mp_poa_set_realign(self.handle))

    def realign_pairs(self, pairs: Sequence[Sequence[np.ndarray]]) -> None:
        """poa_augment with caller pairs: pairs[r] = (matches, gap_x, gap_y) of read r (all
        chunks' reads in order), each (n, 3) int arrays of (weight, x, y)."""
        offs, arrs, keep = [], [], []
        for k in range(3):
            lists = [np.asarray(p[k], dtype=np.int64).reshape(-1, 3) for p in pairs]
            o = np.zeros(len(lists) + 1, dtype=np.int64)
            o[1:] = np.cumsum([a.shape[0] for a in lists])
            a = np.ascontiguousarray(np.concatenate(lists) if lists else np.zeros((1, 3), np.int64))
            if a.size == 0:
                a = np.zeros((1, 3), np.int64)
            keep += [o, a]
            offs.append(_lib.ptr(o, c_int64))
            arrs.append(_lib.ptr(a, c_int64))
        po = (ctypes.POINTER(c_int64) * 3)(*offs)
        pa = (ctypes.POINTER(c_int64) * 3)(*arrs)
        _lib.check(self._lib.mp_poa_set_realign_pairs(self.handle, po, pa))

    def iterate(self) -> None:
        _lib.check(self._lib.mp_poa_set_iterate(self.handle))

    def iterate_polish(self) -> None:
        """poa_realignIterative in polish mode (poa_polish) for every chunk."""
        _lib.check(self._lib.mp_poa_set_iterate_polish(self.handle))

    # ---- the bubble graph of one polish iteration (impl/bubbleGraph.c:800-978) ----
    def build_bubbles(self) -> None:
        _lib.check(self._lib.mp_poa_set_build_bubbles(self.handle))

    def score_bubbles(self) -> None:
        _lib.check(self._lib.mp_poa_set_score_bubbles(self.handle))

    def bubbles(self, chunk: int) -> list:
        """The chunk's bubble graph: per bubble a dict with ref_start, ref_length, alleles (list of
        (chars, counts)), reads ((n, 3) rows of read, start, length), quals and supports
        (alleles x reads, float32)."""
        sz = np.zeros(4, np.int64)
        _lib.check(self._lib.mp_poa_bubble_sizes(self.handle, chunk, _lib.ptr(sz, c_int64)))
        nb, na, runs, nr = (int(v) for v in sz)
        rows = np.zeros((max(nb, 1), 6), np.int64)
        alen = np.zeros(max(na, 1), np.int64)
        chars = (c_char * max(runs, 1))()
        counts = np.zeros(max(runs, 1), np.uint64)
        rd = np.zeros((max(nr, 1), 3), np.int64)
        q = np.zeros(max(nr, 1))
        _lib.check(self._lib.mp_poa_bubbles(self.handle, chunk, _lib.ptr(rows, c_int64), _lib.ptr(alen, c_int64),
                                            chars, _lib.ptr(counts, c_uint64), _lib.ptr(rd, c_int64),
                                            _lib.ptr(q, c_double), None))
        n_sup = int(np.sum(rows[:nb, 3] * rows[:nb, 5]))
        sup = np.zeros(max(n_sup, 1), np.float32)
        _lib.check(self._lib.mp_poa_bubbles(self.handle, chunk, None, None, None, None, None, None,
                                            _lib.ptr(sup, ctypes.c_float)))
        raw = bytes(chars[:runs])
        starts = np.concatenate([[0], np.cumsum(alen[:na])]).astype(np.int64)
        out, at = [], 0
        for i in range(nb):
            rs, rl, af, n_al, rf, n_rd = (int(v) for v in rows[i])
            alleles = [(raw[starts[j]:starts[j + 1]], counts[starts[j]:starts[j + 1]].copy()) for j in range(af, af + n_al)]
            out.append(dict(ref_start=rs, ref_length=rl, alleles=alleles, reads=rd[rf:rf + n_rd].copy(),
                            quals=q[rf:rf + n_rd].copy(), supports=sup[at:at + n_al * n_rd].reshape(n_al, n_rd).copy()))
            at += n_al * n_rd
        return out

    def bubble_consensus(self, chunk: int):
        """(path, consensus RleString, reference-to-consensus map) of the scored bubble graph."""
        sz = np.zeros(4, np.int64)
        _lib.check(self._lib.mp_poa_bubble_sizes(self.handle, chunk, _lib.ptr(sz, c_int64)))
        inf = self.info(chunk)
        cap = 4 * inf["nodes"] + 4 * int(sz[2]) + 16
        path = np.zeros(max(int(sz[0]), 1), np.int64)
        chars = (c_char * cap)()
        counts = np.zeros(cap, np.uint64)
        n = c_int64(0)
        m = np.zeros(max(inf["reference_runs"], 1), np.int64)
        _lib.check(self._lib.mp_poa_bubble_consensus(self.handle, chunk, _lib.ptr(path, c_int64), chars,
                                                     _lib.ptr(counts, c_uint64), cap, ctypes.byref(n),
                                                     _lib.ptr(m, c_int64)))
        return (path[:int(sz[0])].copy(), RleString(bytes(chars[:n.value]), counts[:n.value].astype(np.uint32)),
                m[:inf["reference_runs"]].copy())

    def realign_all(self) -> None:
        _lib.check(self._lib.mp_poa_set_realign_all(self.handle))

    def estimate_repeat_counts(self) -> None:
        _lib.check(self._lib.mp_poa_set_estimate_repeat_counts(self.handle))

    def set_device_steps(self, run_lengths: bool = True, indels: bool = True) -> None:
        """Which steps of a realignment run on the GPU instead of the host threads: the run-length
        estimate and the complete-indel candidates (both on by default); every combination builds
        identical graphs (mp_poa_set_device_steps)."""
        _lib.check(self._lib.mp_poa_set_device_steps(self.handle, (1 if run_lengths else 0) | (2 if indels else 0)))

    PHASES = ("jobs", "device_pass", "fetch", "indel_candidates", "merge", "consensus", "repeat_counts",
              "bubbles", "group", "join")

    def phase_seconds(self) -> dict:
        """Wall seconds spent in each step of the loop since the set was created."""
        v = np.zeros(len(self.PHASES))
        _lib.check(self._lib.mp_poa_set_phase_seconds(self.handle, _lib.ptr(v, c_double), v.size))
        return {k: float(x) for k, x in zip(self.PHASES, v)}

    # ---- inspection ----
    def info(self, chunk: int) -> dict:
        i = _lib.PoaChunkInfo()
        _lib.check(self._lib.mp_poa_info(self.handle, chunk, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in _lib.PoaChunkInfo._fields_}

    def nodes(self, chunk: int) -> dict:
        inf = self.info(chunk)
        n, m = inf["nodes"], inf["max_repeat"]
        bases = (c_char * max(n, 1))()
        rc = np.zeros(n, np.uint64)
        bw = np.zeros((n, 5))
        rcw = np.zeros((n, m))
        no, ni, nd = (np.zeros(n, np.int64) for _ in range(3))
        _lib.check(self._lib.mp_poa_nodes(self.handle, chunk, bases, _lib.ptr(rc, c_uint64), _lib.ptr(bw, c_double),
                                          _lib.ptr(rcw, c_double), _lib.ptr(no, c_int64), _lib.ptr(ni, c_int64),
                                          _lib.ptr(nd, c_int64)))
        return {"bases": bytes(bases[:n]), "repeat_counts": rc, "base_weights": bw, "repeat_count_weights": rcw,
                "n_obs": no, "n_ins": ni, "n_del": nd}

    def observations(self, chunk: int) -> np.ndarray:
        k = self.info(chunk)["observations"]
        r, o, w = np.zeros(k, np.int64), np.zeros(k, np.int64), np.zeros(k)
        _lib.check(self._lib.mp_poa_observations(self.handle, chunk, _lib.ptr(r, c_int64), _lib.ptr(o, c_int64),
                                                 _lib.ptr(w, c_double)))
        return np.stack([r, o, w], axis=1) if k else np.zeros((0, 3))

    def inserts(self, chunk: int) -> list:
        inf = self.info(chunk)
        k, runs = inf["inserts"], inf["insert_runs"]
        wf, wr = np.zeros(k), np.zeros(k)
        ln, no = np.zeros(k, np.int64), np.zeros(k, np.int64)
        chars = (c_char * max(runs, 1))()
        counts = np.zeros(max(runs, 1), np.uint64)
        _lib.check(self._lib.mp_poa_inserts(self.handle, chunk, _lib.ptr(wf, c_double), _lib.ptr(wr, c_double),
                                            _lib.ptr(ln, c_int64), chars, _lib.ptr(counts, c_uint64),
                                            _lib.ptr(no, c_int64)))
        out, at = [], 0
        raw = bytes(chars[:runs])
        for i in range(k):
            out.append((raw[at:at + ln[i]], tuple(int(v) for v in counts[at:at + ln[i]]), float(wf[i]), float(wr[i]),
                        int(no[i])))
            at += int(ln[i])
        return out

    def deletes(self, chunk: int) -> list:
        k = self.info(chunk)["deletes"]
        ln, no = np.zeros(k, np.int64), np.zeros(k, np.int64)
        wf, wr = np.zeros(k), np.zeros(k)
        _lib.check(self._lib.mp_poa_deletes(self.handle, chunk, _lib.ptr(ln, c_int64), _lib.ptr(wf, c_double),
                                            _lib.ptr(wr, c_double), _lib.ptr(no, c_int64)))
        return [(int(ln[i]), float(wf[i]), float(wr[i]), int(no[i])) for i in range(k)]

    def reference(self, chunk: int) -> RleString:
        n = self.info(chunk)["reference_runs"]
        chars = (c_char * max(n, 1))()
        counts = np.zeros(max(n, 1), np.uint64)
        _lib.check(self._lib.mp_poa_reference(self.handle, chunk, chars, _lib.ptr(counts, c_uint64)))
        return RleString(bytes(chars[:n]), counts[:n].astype(np.uint32))

    def consensus(self, chunk: int):
        """(consensus RleString, node-to-consensus map)."""
        inf = self.info(chunk)
        cap = 4 * inf["nodes"] + 16 * (inf["insert_runs"] + 1)
        chars = (c_char * cap)()
        counts = np.zeros(cap, np.uint64)
        n = c_int64(0)
        m = np.zeros(max(inf["nodes"] - 1, 1), np.int64)
        _lib.check(self._lib.mp_poa_consensus(self.handle, chunk, chars, _lib.ptr(counts, c_uint64), cap, n,
                                              _lib.ptr(m, c_int64)))
        return RleString(bytes(chars[:n.value]), counts[:n.value].astype(np.uint32)), m[:inf["nodes"] - 1].copy()

    def anchor_alignments(self, chunk: int, node_map: Optional[np.ndarray] = None) -> List[np.ndarray]:
        nr = self.reads_per_chunk[chunk]
        inf = self.info(chunk)
        cap = inf["observations"] + 1
        offs = np.zeros(nr + 1, np.int64)
        tri = np.zeros((cap, 3), np.int64)
        n = c_int64(0)
        mp = None if node_map is None else np.ascontiguousarray(node_map, dtype=np.int64)
        _lib.check(self._lib.mp_poa_anchor_alignments(self.handle, chunk, _lib.ptr(mp, c_int64),
                                                      _lib.ptr(offs, c_int64), _lib.ptr(tri, c_int64), cap, n))
        return [tri[offs[r]:offs[r + 1]].copy() for r in range(nr)]

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.mp_poa_set_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def polish(engine: Engine, model: Model, pm: PolishModel, polish_params: PolishParams, drafts, reads, strands,
           anchors=None, qualities=None) -> List[RleString]:
    """poa_realignAll for every chunk (the consensus iterations, then the polish iterations, as
    polish_params sets them), then the run-length estimate the caller applies to the result
    (marginPolish.c:554-560): each chunk's polished draft."""
    s = PoaSet.from_polish_model(engine, model, pm, polish_params, drafts, reads, strands, anchors, qualities)
    try:
        s.realign_all()
        if polish_params.use_run_length:
            s.estimate_repeat_counts()
        return [s.reference(c) for c in range(s.n_chunks)]
    finally:
        s.close()


def merge_contig(engine: Engine, model: Model, params: AlignmentParams, chunks: Sequence[str], overlap: int,
                 spacer_length: Optional[int] = None):
    """mergeContigChunks (impl/chunker.c:50-112): the polished chunks of one contig (expanded
    strings, in order) joined at their overlaps, each boundary cut by removeOverlap
    (impl/polisher.c:1937-2006) with `model` (the reference uses the code-default nucleotide
    machine, params.code_default_state_model()). overlap is twice the chunk boundary
    (marginPolish.c:658); the spacer for a missing chunk is 3 x the chunk boundary Ns (50 with
    no boundary, marginPolish.c:639). Returns (merged string, report rows of (boundary weight,
    characters cut from the chunk's start, 1 spacer / 2 seam of Ns / 0))."""
    if spacer_length is None:
        spacer_length = 50 if overlap == 0 else 3 * (overlap // 2)
    raw = [c.encode() for c in chunks]
    off = np.zeros(len(raw) + 1, np.int64)
    off[1:] = np.cumsum([len(c) for c in raw])
    flat = b"".join(raw) or b"\0"
    cap = int(off[-1]) + spacer_length * len(raw) + 10 * len(raw) + 16
    out = (c_char * cap)()
    n = c_int64(0)
    report = np.zeros((max(len(raw), 1), 3), np.int64)
    ps = params.struct()
    _lib.check(engine._lib.mp_merge_contig(engine.handle, model.handle, ctypes.byref(ps), len(raw),
                                           _lib.ptr(off, c_int64), flat, int(overlap), int(spacer_length), out, cap,
                                           ctypes.byref(n), _lib.ptr(report, c_int64)))
    return bytes(out[:n.value]).decode(), report[:len(raw)].copy()

def merge_contig_threaded(engine: Engine, model: Model, params: AlignmentParams, chunks: Sequence[str],
                          overlap: int, groups: int, spacer_length: Optional[int] = None) -> str:
    """mergeContigChunksThreaded (impl/chunker.c:114-152): the chunks split into `groups` runs of
    ceil(n / groups) (fewer groups when the last would be empty), each run merged, then the
    merged runs merged with the same overlap. One GPU call per run (each already batches its
    boundaries), one for the runs."""
    n = len(chunks)
    if groups <= 1 or n == 0:
        return merge_contig(engine, model, params, chunks, overlap, spacer_length)[0]
    per = -(-n // groups)
    while per * (groups - 1) >= n:
        groups -= 1
    runs = [merge_contig(engine, model, params, chunks[g * per:min(n, (g + 1) * per)], overlap, spacer_length)[0]
            for g in range(groups)]
    return merge_contig(engine, model, params, runs, overlap, spacer_length)[0]


def node_update(engine: Engine, drafts: Sequence[RleString], reads: Sequence[Sequence[RleString]],
                strands: Sequence[Sequence[int]], matches: Sequence[np.ndarray], max_repeat: int,
                repeat_log10: Optional[np.ndarray] = None, observations: bool = True) -> dict:
    """The device-side node update (mp_node_update) of one graph per draft: the match part of
    poa_augment (impl/polisher.c:322-340) and the run-length estimate (:1556-1565, :1796-1865).
    matches[r] is the (n, 3) (weight, x, y) match list of read r (all chunks' reads in order).
    Returns per chunk the base weights, run-length weights, observations (read, offset, weight) in
    poa_augment's order and, with repeat_log10, the estimated run length of every node."""
    lib = engine._lib
    n_chunks = len(drafts)
    node_off = np.zeros(n_chunks + 1, dtype=np.int64)
    node_off[1:] = np.cumsum([len(d) + 1 for d in drafts])
    bases = b"".join(b"N" + bytes(b if chr(b) in "ACGT" else ord("N") for b in d.chars.upper()) for d in drafts)
    flat = [r for lst in reads for r in lst]
    chunk_reads = np.zeros(n_chunks + 1, dtype=np.int64)
    chunk_reads[1:] = np.cumsum([len(lst) for lst in reads])
    rd_off, rd_chars, rd_counts = _flat_rle(flat)
    strand = np.ascontiguousarray([int(s) for lst in strands for s in lst], dtype=np.uint8)
    if strand.size != len(flat) or len(matches) != len(flat):
        raise ValueError("one strand and one match list per read")
    lists = [np.asarray(m, dtype=np.int64).reshape(-1, 3) for m in matches]
    m_off = np.zeros(len(lists) + 1, dtype=np.int64)
    m_off[1:] = np.cumsum([a.shape[0] for a in lists])
    allm = np.concatenate(lists) if lists else np.zeros((0, 3), np.int64)
    w = np.ascontiguousarray(allm[:, 0], dtype=np.int32)
    x = np.ascontiguousarray(allm[:, 1], dtype=np.int32)
    y = np.ascontiguousarray(allm[:, 2], dtype=np.int32)
    rep = None if repeat_log10 is None else np.ascontiguousarray(repeat_log10, dtype=np.float64).reshape(-1)
    b = _lib.NodeBatch()
    b.n_chunks = n_chunks
    b.node_offsets = _lib.ptr(node_off, c_int64)
    bases_buf = ctypes.create_string_buffer(bases, max(len(bases), 1))
    b.node_bases = ctypes.cast(bases_buf, ctypes.POINTER(c_char))
    b.chunk_reads = _lib.ptr(chunk_reads, c_int64)
    b.read_offsets = _lib.ptr(rd_off, c_int64)
    chars_buf = ctypes.create_string_buffer(rd_chars or b"\0", max(len(rd_chars), 1))
    b.read_chars = ctypes.cast(chars_buf, ctypes.POINTER(c_char))
    b.read_counts = _lib.ptr(rd_counts if rd_counts.size else np.zeros(1, np.uint32), c_uint32)
    b.strand = _lib.ptr(strand if strand.size else np.zeros(1, np.uint8), c_uint8)
    b.match_offsets = _lib.ptr(m_off, c_int64)
    b.weight = _lib.ptr(w if w.size else np.zeros(1, np.int32), c_int32)
    b.x = _lib.ptr(x if x.size else np.zeros(1, np.int32), c_int32)
    b.y = _lib.ptr(y if y.size else np.zeros(1, np.int32), c_int32)
    b.max_repeat = int(max_repeat)
    b.repeat_log10 = _lib.ptr(rep, c_double)
    n_nodes, n_tup = int(node_off[-1]), int(m_off[-1])
    bw = np.zeros((max(n_nodes, 1), 5))
    rcw = np.zeros((max(n_nodes, 1), int(max_repeat)))
    obs_off = np.zeros(n_nodes + 1, dtype=np.int64)
    o_read, o_off = np.zeros(max(n_tup, 1), np.int64), np.zeros(max(n_tup, 1), np.int64)
    o_w = np.zeros(max(n_tup, 1))
    rc = np.zeros(max(n_nodes, 1), np.uint64)
    r = _lib.NodeResult()
    r.base_weights = _lib.ptr(bw, c_double)
    r.repeat_weights = _lib.ptr(rcw, c_double)
    r.obs_offsets = _lib.ptr(obs_off, c_int64)
    if observations:
        r.obs_read = _lib.ptr(o_read, c_int64)
        r.obs_offset = _lib.ptr(o_off, c_int64)
        r.obs_weight = _lib.ptr(o_w, c_double)
    if rep is not None:
        r.repeat_counts = _lib.ptr(rc, c_uint64)
    _lib.check(lib.mp_node_update(engine.handle, ctypes.byref(b), ctypes.byref(r)))
    out = []
    for c in range(n_chunks):
        g0, g1 = int(node_off[c]), int(node_off[c + 1])
        o0, o1 = int(obs_off[g0]), int(obs_off[g1])
        d = {"base_weights": bw[g0:g1].copy(), "repeat_count_weights": rcw[g0:g1].copy(),
             "n_obs": np.diff(obs_off[g0:g1 + 1])}
        if observations:
            d["observations"] = np.stack([o_read[o0:o1], o_off[o0:o1], o_w[o0:o1]], axis=1) if o1 > o0 \
                else np.zeros((0, 3))
        if rep is not None:
            d["repeat_counts"] = rc[g0 + 1:g1].copy()
        out.append(d)
    return {"chunks": out}
