"""Seeded synthetic workloads for the realignment pass.

Stands in for BAM input (no reads or genomes ship with this project): a
template (draft) per chunk, reads sampled from it with a nanopore-like error
model, their base-level truth alignment turned into run-length anchors exactly
as MarginPolish turns CIGAR match positions into anchors
(impl/htsIntegration.c:493-499 tuples, runLengthEncodeAlignment
impl/polisher.c:1732-1750), and the per-read reference crop of
getAlignedPairsWithIndelsCroppingReference (impl/polisher.c:613-628).

Error model: homopolymer run length perturbed by +-1 (p=0.15) or +-2
(p=0.03), then per base: deletion 5%, substitution 3%, insertion after the
base 4%. Generator: numpy PCG64 with the given seed.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .realign import Jobs
from .rle import RleString, crop_range, rle_anchors

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)


@dataclass
class ErrorModel:
    sub: float = 0.03
    ins: float = 0.04
    dele: float = 0.05
    hp1: float = 0.15
    hp2: float = 0.03


@dataclass
class Workload:
    """Templates, reads and anchors of one synthetic configuration."""

    name: str
    templates: List[RleString]
    reads: List[RleString]
    read_template: np.ndarray        # template index of each read
    strand: np.ndarray               # 1 forward
    anchors: List[np.ndarray]        # per read, RLE anchors in full-template coordinates (x, y, expansion)
    expansion: int
    meta: dict = field(default_factory=dict)

    def jobs(self, max_repeat_exclusive: int = 51, include_counts: bool = True) -> Jobs:
        """Cropped jobs exactly as poa_realign hands them to the aligner."""
        tsyms = [t.symbols(include_counts, max_repeat_exclusive) for t in self.templates]
        toff = np.zeros(len(tsyms) + 1, dtype=np.int64)
        toff[1:] = np.cumsum([s.size for s in tsyms])
        xs = np.concatenate(tsyms) if tsyms else np.zeros(0, np.uint16)
        n = len(self.reads)
        xb = np.zeros(n, np.int64)
        xe = np.zeros(n, np.int64)
        shift = np.zeros(n, np.int64)
        ys_list, an_list = [], []
        yoff = np.zeros(n + 1, np.int64)
        aoff = np.zeros(n + 1, np.int64)
        for i, (r, a, t) in enumerate(zip(self.reads, self.anchors, self.read_template)):
            s, e = crop_range(a, len(self.templates[t]), len(r))
            xb[i] = toff[t] + s
            xe[i] = toff[t] + e
            shift[i] = s
            aa = a.copy()
            aa[:, 0] -= s
            an_list.append(aa)
            ys_list.append(r.symbols(include_counts, max_repeat_exclusive))
            yoff[i + 1] = yoff[i] + ys_list[-1].size
            aoff[i + 1] = aoff[i] + aa.shape[0]
        ys = np.concatenate(ys_list) if ys_list else np.zeros(0, np.uint16)
        an = np.concatenate(an_list) if an_list else np.zeros((0, 3), np.int32)
        return Jobs(xs, xb, xe, ys, yoff, an, aoff, self.strand.astype(np.uint8), None, None, shift)


def random_template(rng: np.random.Generator, length: int, gc: float = 0.5, run_p: Optional[float] = None,
                    run_cap: int = 20) -> np.ndarray:
    """uint8 ASCII bases. run_p=None: i.i.d. bases; otherwise runs with geometric(run_p) lengths capped at run_cap,
    consecutive runs of different bases, base composition with the given GC fraction."""
    probs = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    if run_p is None:
        return BASES[rng.choice(4, size=length, p=probs)]
    nruns = int(length / (1.0 / run_p) * 1.3) + 16
    lens = np.minimum(rng.geometric(run_p, size=nruns), run_cap)
    b = rng.choice(4, size=nruns, p=probs)
    # force consecutive runs to differ: resample equal neighbours by rotating
    for _ in range(8):
        same = np.nonzero(b[1:] == b[:-1])[0] + 1
        if same.size == 0:
            break
        b[same] = (b[same] + rng.integers(1, 4, size=same.size)) % 4
    seq = np.repeat(BASES[b], lens)
    while seq.size < length:
        seq = np.concatenate([seq, random_template(rng, length - seq.size, gc, run_p, run_cap)])
    return seq[:length]


def mutate_read(rng: np.random.Generator, seg: np.ndarray, em: ErrorModel):
    """Returns (read bytes, truth pairs (template index within seg, read index)) for a template segment."""
    n = seg.size
    # run-length decomposition of the segment
    brk = np.nonzero(seg[1:] != seg[:-1])[0] + 1
    starts = np.concatenate([[0], brk])
    counts = np.diff(np.concatenate([starts, [n]]))
    u = rng.random(counts.size)
    sign = np.where(rng.random(counts.size) < 0.5, -1, 1)
    delta = np.where(u < em.hp2, 2, np.where(u < em.hp2 + em.hp1, 1, 0)) * sign
    rcounts = np.maximum(1, counts + delta)
    # read core: bases of each run, aligned pairwise up to min(count, rcount)
    run_of = np.repeat(np.arange(counts.size), rcounts)
    core_start = np.concatenate([[0], np.cumsum(rcounts)[:-1]])
    idx_in_run = np.arange(run_of.size) - core_start[run_of]
    core_bases = seg[starts[run_of]]
    aligned = idx_in_run < counts[run_of]
    tpos = starts[run_of] + idx_in_run
    # per-base errors
    m = core_bases.size
    keep = rng.random(m) >= em.dele
    sub = (rng.random(m) < em.sub) & keep
    ins = rng.random(m) < em.ins
    out_bases = core_bases.copy()
    if sub.any():
        cur = np.searchsorted(BASES, out_bases[sub])
        out_bases[sub] = BASES[(cur + rng.integers(1, 4, size=int(sub.sum()))) % 4]
    per = keep.astype(np.int64) + ins.astype(np.int64)
    pos = np.concatenate([[0], np.cumsum(per)[:-1]])
    total = int(per.sum())
    read = np.empty(total, dtype=np.uint8)
    read[pos[keep]] = out_bases[keep]
    ins_pos = pos[ins] + keep[ins].astype(np.int64)
    read[ins_pos] = BASES[rng.integers(0, 4, size=int(ins.sum()))]
    ok = keep & aligned
    pairs = np.stack([tpos[ok], pos[ok]], axis=1)
    return read, pairs


def sample_reads(rng, template: np.ndarray, n_reads: int, length_sampler, em: ErrorModel):
    out = []
    L = template.size
    for _ in range(n_reads):
        ln = int(min(max(length_sampler(), 64), L))
        off = int(rng.integers(0, L - ln + 1))
        read, pairs = mutate_read(rng, template[off:off + ln], em)
        pairs[:, 0] += off
        out.append((read, pairs, int(rng.integers(0, 2))))
    return out


def build_workload(name: str, rng, templates_ascii: List[np.ndarray], reads_per_template: List[list],
                   expansion: int, meta: dict) -> Workload:
    templates = [RleString.from_string(t.tobytes()) for t in templates_ascii]
    reads, anchors, rt, strand = [], [], [], []
    for ti, lst in enumerate(reads_per_template):
        for read, pairs, s in lst:
            r = RleString.from_string(read.tobytes())
            p = np.concatenate([pairs, np.full((pairs.shape[0], 1), expansion, dtype=np.int64)], axis=1)
            a = rle_anchors(p, templates[ti], r)
            if a.shape[0] == 0 or len(r) == 0:
                continue
            reads.append(r)
            anchors.append(a)
            rt.append(ti)
            strand.append(s)
    return Workload(name, templates, reads, np.array(rt, dtype=np.int64), np.array(strand, dtype=np.uint8),
                    anchors, expansion, meta)


def config_small(seed: int = 1, n_reads: int = 20, template_len: int = 2000, half_width: int = 25) -> Workload:
    """One chunk: 2 kb i.i.d. template, 20 reads of 1.5-2 kb, band half-width 25 (expansion 50)."""
    rng = np.random.default_rng(seed)
    em = ErrorModel()
    t = random_template(rng, template_len)
    reads = sample_reads(rng, t, n_reads, lambda: rng.integers(1500, 2001), em)
    return build_workload("small", rng, [t], [reads], 2 * half_width,
                          {"template_bp": template_len, "reads": n_reads, "half_width": half_width})


def config_batched(seed: int = 2, n_chunks: int = 256, chunk_len: int = 10_000, coverage: float = 30.0,
                   median: float = 6000.0, sigma: float = 0.6, half_width: int = 25) -> Workload:
    """Uneven batch: chunks of homopolymer-enriched templates (GC 0.41, runs geometric p=0.55 capped 20),
    log-normal read lengths truncated to the chunk."""
    rng = np.random.default_rng(seed)
    em = ErrorModel()
    mean_len = min(float(chunk_len), median * float(np.exp(sigma ** 2 / 2)))
    templates, per = [], []
    for _ in range(n_chunks):
        t = random_template(rng, chunk_len, gc=0.41, run_p=0.55, run_cap=20)
        n = max(1, int(round(coverage * chunk_len / mean_len)))
        per.append(sample_reads(rng, t, n, lambda: rng.lognormal(np.log(median), sigma), em))
        templates.append(t)
    return build_workload("batched", rng, templates, per, 2 * half_width,
                          {"chunks": n_chunks, "chunk_bp": chunk_len, "coverage": coverage, "half_width": half_width})


def config_adjoint(seed: int = 4, n_reads: int = 512, n_templates: int = 64, template_len: int = 5000,
                   half_width: int = 25) -> Workload:
    """512 reads of 2-5 kb on 64 random 5 kb templates."""
    rng = np.random.default_rng(seed)
    em = ErrorModel()
    templates = [random_template(rng, template_len) for _ in range(n_templates)]
    per = [[] for _ in range(n_templates)]
    for i in range(n_reads):
        ti = i % n_templates
        per[ti] += sample_reads(rng, templates[ti], 1, lambda: rng.integers(2000, 5001), em)
    return build_workload("adjoint", rng, templates, per, 2 * half_width,
                          {"reads": n_reads, "templates": n_templates, "half_width": half_width})


def config_by_name(name: str, **kw) -> Workload:
    return {"small": config_small, "batched": config_batched, "adjoint": config_adjoint}[name](**kw)
