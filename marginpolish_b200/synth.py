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

The generator's integer steps (run-length encoding, symbols, run-length anchors,
reference crop) are numpy restatements of the same reference rules, so that
building a workload maps no native library: the reference arm of the benchmark
generates its inputs without loading the CUDA library. tests/test_rle.py checks
them bit-exact against the library's routines.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .realign import Jobs
from .rle import RleString

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)

# nucleotide alphabet of impl/stateMachine.c:25-42 ('N' and every other character -> 4)
_SYMBOL_OF = np.full(256, 4, dtype=np.uint16)
for _c, _v in zip(b"ACGTacgt", (0, 1, 2, 3, 0, 1, 2, 3)):
    _SYMBOL_OF[_c] = _v


def rle_encode(seq) -> RleString:
    """rleString_construct (impl/polisher.c:1357-1389): one run per maximal stretch of equal
    characters (case-sensitive)."""
    a = np.frombuffer(bytes(seq), dtype=np.uint8) if not isinstance(seq, np.ndarray) else seq.astype(np.uint8)
    if a.size == 0:
        return RleString(b"", np.zeros(0, dtype=np.uint32))
    ends = np.concatenate([np.nonzero(a[1:] != a[:-1])[0], [a.size - 1]])
    starts = np.concatenate([[0], ends[:-1] + 1])
    return RleString(a[ends].tobytes(), (ends - starts + 1).astype(np.uint32))


def rle_symbols(r: RleString, include_counts: bool = True, max_repeat_exclusive: int = 51) -> np.ndarray:
    """rleString_constructSymbolString (impl/stateMachine.c:133-146): base symbol, and the run
    length clamped to max_repeat_exclusive - 1 in the high byte (symbol_addRepeatCount, :124-131)."""
    b = _SYMBOL_OF[np.frombuffer(r.chars, dtype=np.uint8)]
    if include_counts:
        rc = np.minimum(r.counts.astype(np.int64), max_repeat_exclusive - 1).astype(np.uint16)
        b = (rc << np.uint16(8)) | b
    return b.astype(np.uint16)


def _run_ends(v: np.ndarray) -> np.ndarray:
    """For a non-decreasing array: per element, the index of the first element greater than it."""
    step = v[1:] != v[:-1]
    ends = np.append(np.flatnonzero(step) + 1, v.size)
    run = np.concatenate([[0], np.cumsum(step)])
    return ends[run]


def rle_anchors_monotone(pairs: np.ndarray, x: RleString, y: RleString, xmap: Optional[np.ndarray] = None,
                         ymap: Optional[np.ndarray] = None) -> np.ndarray:
    """runLengthEncodeAlignment (impl/polisher.c:1732-1750) for base pairs strictly increasing in
    both coordinates: each pair goes through the non-RLE -> RLE coordinate maps (:1718-1730; xmap /
    ymap may be passed in precomputed) and is kept when both RLE coordinates exceed the last kept
    pair's. The mapped coordinates are then non-decreasing, so the pair kept after pair i is the
    first j with x2[j] > x2[i] and y2[j] > y2[i], i.e. the later of the ends of the runs of equal
    x2 and of equal y2 that hold i; the kept pairs are the orbit of pair 0 under that successor
    map, found by doubling (the orbit is increasing, so it comes out in order)."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 3)
    m = pairs.shape[0]
    if m == 0:
        return np.zeros((0, 3), dtype=np.int32)
    if np.any(np.diff(pairs[:, 0]) <= 0) or np.any(np.diff(pairs[:, 1]) <= 0):
        raise ValueError("base pairs must be strictly increasing in both coordinates")
    if xmap is None:
        xmap = np.repeat(np.arange(len(x), dtype=np.int64), x.counts.astype(np.int64))
    if ymap is None:
        ymap = np.repeat(np.arange(len(y), dtype=np.int64), y.counts.astype(np.int64))
    x2 = xmap[pairs[:, 0]]
    y2 = ymap[pairs[:, 1]]
    succ = np.empty(m + 1, dtype=np.int64)
    succ[:m] = np.maximum(_run_ends(x2), _run_ends(y2))
    succ[m] = m  # sink
    orbit = np.zeros(1, dtype=np.int64)
    step = succ
    while orbit[-1] < m:
        orbit = np.concatenate([orbit, step[orbit]])  # the next len(orbit) members
        step = step[step]
    keep = orbit[orbit < m]
    return np.stack([x2[keep], y2[keep], pairs[keep, 2]], axis=1).astype(np.int32)


def crop_range(anchors: np.ndarray, template_length: int, read_length: int) -> tuple:
    """Template crop of getAlignedPairsWithIndelsCroppingReference (impl/polisher.c:613-628):
    [max(0, x0 - y0), min(lX, 1 + xN + (lY - yN)))."""
    a = np.asarray(anchors, dtype=np.int64).reshape(-1, 3)
    if a.shape[0] == 0:
        return 0, int(template_length)
    s = max(0, int(a[0, 0] - a[0, 1]))
    e = min(int(template_length), int(1 + a[-1, 0] + (read_length - a[-1, 1])))
    if s >= template_length or e < 0:
        raise ValueError("crop range outside the template")
    return s, e


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
        tsyms = [rle_symbols(t, include_counts, max_repeat_exclusive) for t in self.templates]
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
            ys_list.append(rle_symbols(r, include_counts, max_repeat_exclusive))
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
    templates = [rle_encode(t) for t in templates_ascii]
    reads, anchors, rt, strand = [], [], [], []
    for ti, lst in enumerate(reads_per_template):
        for read, pairs, s in lst:
            r = rle_encode(read)
            p = np.concatenate([pairs, np.full((pairs.shape[0], 1), expansion, dtype=np.int64)], axis=1)
            a = rle_anchors_monotone(p, templates[ti], r)
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


def config_long_reads(seed: int, lengths, half_width: int, template_len: int = 160_000) -> Workload:
    """Reads of the given base lengths sampled from one homopolymer-enriched template (GC 0.5,
    geometric run lengths p = 0.55, capped at 20) with the nanopore-like error model, anchors of
    band half-width `half_width` (the long reads of the polishing configurations at scale)."""
    rng = np.random.default_rng(seed)
    em = ErrorModel()
    t = random_template(rng, template_len, gc=0.5, run_p=0.55, run_cap=20)
    lst = []
    for ln in lengths:
        ln = int(min(ln, t.size))
        off = int(rng.integers(0, t.size - ln + 1))
        read, pairs = mutate_read(rng, t[off:off + ln], em)
        pairs[:, 0] += off
        lst.append((read, pairs, int(rng.integers(0, 2))))
    return build_workload("long_reads", rng, [t], [lst], 2 * half_width,
                          {"template_bp": template_len, "read_bp": [int(v) for v in lengths],
                           "half_width": half_width})


def draft_with_errors(rng: np.random.Generator, truth: np.ndarray, rate: float = 0.01, hp_bias: float = 0.7):
    """A draft assembly: the truth with indels at `rate` per base, a fraction hp_bias of them
    lengthening or shortening a homopolymer run by one base, the rest single-base indels
    at random positions. Returns (draft bytes, base pairs (truth index, draft index))."""
    n = truth.size
    brk = np.nonzero(truth[1:] != truth[:-1])[0] + 1
    starts = np.concatenate([[0], brk])
    counts = np.diff(np.concatenate([starts, [n]]))
    n_err = int(rng.binomial(n, rate))
    ops = {}  # truth index -> 'd' (drop) or inserted base (insert after)
    long_runs = starts[counts >= 2]
    for _ in range(n_err):
        if rng.random() < hp_bias and long_runs.size:
            st = int(rng.choice(long_runs))
            ops[st] = "d" if rng.random() < 0.5 else truth[st]
        else:
            i = int(rng.integers(0, n))
            ops[i] = "d" if rng.random() < 0.5 else BASES[int(rng.integers(0, 4))]
    out, pairs = [], []
    for i in range(n):
        op = ops.get(i)
        if op == "d":
            continue
        pairs.append((i, len(out)))
        out.append(truth[i])
        if op is not None:
            out.append(op)
    return np.array(out, dtype=np.uint8), np.array(pairs, dtype=np.int64).reshape(-1, 2)


@dataclass
class PolishWorkload:
    """Chunks for the POA loop: per chunk the truth, the draft (RLE) and the reads (RLE, strand,
    anchors against the draft in RLE coordinates)."""
    truths: List[RleString]
    drafts: List[RleString]
    reads: List[List[RleString]]
    strands: List[List[int]]
    anchors: List[List[np.ndarray]]
    meta: dict = field(default_factory=dict)

    def qualities(self, seed: int = 0, mean=(12.0, 3.0), spread: float = 4.0) -> List[List[np.ndarray]]:
        """Seeded nanopore-like base qualities in the run-length form the reference keeps
        (rleString_rleQualities, impl/polisher.c:1692-1714: each run gets the integer mean of
        its bases' qualities): per read a phred level drawn from N(mean), per base that level
        plus N(0, spread), clipped to [2, 40]."""
        rng = np.random.default_rng(seed)
        out = []
        for chunk in self.reads:
            lst = []
            for r in chunk:
                counts = np.asarray(r.counts, dtype=np.int64)
                level = float(np.clip(rng.normal(mean[0], mean[1]), 4.0, 30.0))
                q = np.clip(np.rint(rng.normal(level, spread, size=int(counts.sum()))), 2, 40).astype(np.int64)
                starts = np.concatenate([[0], np.cumsum(counts)[:-1]]) if counts.size else np.zeros(0, np.int64)
                sums = np.add.reduceat(q, starts) if counts.size else np.zeros(0, np.int64)
                lst.append((sums // np.maximum(counts, 1)).astype(np.uint8))
            out.append(lst)
        return out

    def realign_workload(self) -> Workload:
        """The first realignment of the polishing loop as a plain workload: every read of every
        chunk against its chunk's draft with its anchors (poa_realign, impl/polisher.c:656-703)."""
        reads, anchors, rt, strand = [], [], [], []
        for c in range(len(self.drafts)):
            for r, s, a in zip(self.reads[c], self.strands[c], self.anchors[c]):
                reads.append(r)
                anchors.append(a)
                rt.append(c)
                strand.append(s)
        exp = int(anchors[0][0, 2]) if anchors and anchors[0].shape[0] else 0
        return Workload("realign", list(self.drafts), reads, np.array(rt, dtype=np.int64),
                        np.array(strand, dtype=np.uint8), anchors, exp, dict(self.meta))


def config_polish(seed: int = 3, n_chunks: int = 1, chunk_len: int = 2000, coverage: float = 20.0,
                  read_len=(1500, 2000), half_width: int = 25, draft_error: float = 0.01,
                  hp_runs: bool = False, read_lognormal=None) -> PolishWorkload:
    """Polishing chunks: truth templates, drafts = truth with 1% homopolymer-biased indels,
    reads sampled from the truth with the nanopore-like error model, anchors from the reads'
    truth alignment carried through the truth-to-draft map (every aligned base, expansion
    2 * half_width, then run-length encoded as CIGAR anchors are). Read lengths are uniform in
    read_len, or log-normal when read_lognormal = (median, sigma, maximum) is given."""
    rng = np.random.default_rng(seed)
    em = ErrorModel()
    truths, drafts, reads, strands, anchors = [], [], [], [], []
    for _ in range(n_chunks):
        t = random_template(rng, chunk_len, gc=0.41 if hp_runs else 0.5, run_p=0.55 if hp_runs else None)
        d, t2d = draft_with_errors(rng, t, draft_error)
        tmap = np.full(t.size, -1, dtype=np.int64)
        tmap[t2d[:, 0]] = t2d[:, 1]
        drle = rle_encode(d)
        dmap = np.repeat(np.arange(len(drle), dtype=np.int64), drle.counts.astype(np.int64))
        if read_lognormal is not None:
            med, sig, mx = read_lognormal
            mean_len = min(float(mx), float(med) * float(np.exp(sig ** 2 / 2)))
            draw = lambda: int(min(mx, rng.lognormal(np.log(med), sig)))  # noqa: E731
        else:
            mean_len = float(np.mean(read_len))
            draw = lambda: int(rng.integers(read_len[0], read_len[1] + 1))  # noqa: E731
        n_reads = max(1, int(round(coverage * chunk_len / mean_len)))
        # reads overhang the chunk ends and are clipped to it (as the chunker clips alignments),
        # so the coverage is even up to the chunk's ends
        lst = []
        for _ in range(n_reads):
            ln = max(64, draw())
            start = int(rng.integers(-ln // 2, t.size - ln // 2))
            a, b = max(0, start), min(t.size, start + ln)
            if b - a < 64:
                continue
            read, pairs = mutate_read(rng, t[a:b], em)
            pairs[:, 0] += a
            lst.append((read, pairs, int(rng.integers(0, 2))))
        cr, cs, ca = [], [], []
        for read, pairs, s in lst:
            r = rle_encode(read)
            dp = tmap[pairs[:, 0]]
            ok = dp >= 0
            p = np.stack([dp[ok], pairs[ok, 1], np.full(int(ok.sum()), 2 * half_width)], axis=1)
            a = rle_anchors_monotone(p, drle, r, xmap=dmap)
            if a.shape[0] == 0 or len(r) == 0:
                continue
            cr.append(r)
            cs.append(s)
            ca.append(a)
        truths.append(rle_encode(t))
        drafts.append(drle)
        reads.append(cr)
        strands.append(cs)
        anchors.append(ca)
    return PolishWorkload(truths, drafts, reads, strands, anchors,
                          {"chunks": n_chunks, "chunk_bp": chunk_len, "coverage": coverage, "half_width": half_width,
                           "draft_error": draft_error})


def config_by_name(name: str, **kw) -> Workload:
    return {"small": config_small, "batched": config_batched, "adjoint": config_adjoint}[name](**kw)
