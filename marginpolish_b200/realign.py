"""Host-side interface of the realignment pass, mirroring the reference's
operator API for this path:

* ``get_aligned_pairs_with_indels_using_anchors`` -- getAlignedPairsWithIndelsUsingAnchors
  (impl/pairwiseAligner.c:1105-1130): match, gap-x and gap-y posterior tuples
  (weight, x, y) of one read, in the reference's output order;
* ``get_aligned_pairs_using_anchors`` -- getAlignedPairsUsingAnchors (:1088-1103);
* ``get_aligned_pairs_with_indels_cropping_reference`` -- the per-read call of
  poa_realign (impl/polisher.c:605-654), including the reference crop and the
  gap-x -> deletes / gap-y -> inserts naming;
* ``realign_batch`` -- all reads of all chunks in one call (the batched form
  poa_realignAll's per-read loop maps onto);
* ``compute_forward_probability`` / ``forward_batch`` -- computeForwardProbability
  (impl/pairwiseAligner.c:813-865), the forward log-likelihood the bubble graph
  scores alleles with (impl/bubbleGraph.c:924);
* ``expectations_batch`` -- expected counts of transitions and emissions, i.e. the
  gradient of the summed log-likelihood with respect to the log parameters
  (the Baum-Welch counts of getExpectationsUsingAnchors, :1151-1156).

Every call goes through the CUDA library (libmpgpu.so); errors of the C ABI
are raised as MpError.
"""
from __future__ import annotations

import ctypes
import weakref
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import c_float, c_int32, c_int64, c_uint8, c_uint16, c_void_p
from .params import AlignmentParams, PolishModel, StateModel


class Engine:
    """One CUDA device (one process per GPU)."""

    def __init__(self, device: int = 0):
        self._lib = _lib.load()
        h = c_void_p()
        _lib.check(self._lib.mp_engine_create(device, ctypes.byref(h)))
        self.handle = h
        sm, ma, mi = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self._lib.mp_engine_info(h, sm, ma, mi))
        self.sm_count, self.cc = sm.value, (ma.value, mi.value)

    def set_tuning(self, warps_per_block: int = 0, blocks_per_sm: int = 0, lanes_per_task: int = 0) -> None:
        """Posterior-kernel tuning (0 = automatic): resident warps per block, persistent blocks
        per SM, and lanes per banded sub-problem (32, 16 or 8)."""
        t = _lib.Tuning(0, warps_per_block, blocks_per_sm, lanes_per_task)
        _lib.check(self._lib.mp_engine_set_tuning(self.handle, ctypes.byref(t)))

    def autotune(self, model: "Model", params, sample: "Jobs") -> list:
        """Times the FP32 kernel variants (band tile shape, checkpoint stride) and warps per
        block on the sub-problems of `sample` per band-hull class and makes the fastest the
        engine's choice (mp_engine_autotune). Returns one dict per class."""
        rep = _lib.AutotuneReport()
        p = params.struct() if hasattr(params, "struct") else params
        _lib.check(self._lib.mp_engine_autotune(self.handle, model.handle, ctypes.byref(p),
                                                ctypes.byref(sample.struct()), ctypes.byref(rep)))
        out = []
        for c in range(rep.n_classes):
            out.append({k: (float(getattr(rep, k)[c]) if k.endswith("gcups") else int(getattr(rep, k)[c]))
                        for k in ("max_hull", "tasks", "candidates", "variant", "lanes_per_task", "cells_per_lane",
                                  "checkpoint_stride", "warps_per_block", "gcups", "default_gcups")})
        return out

    def set_graph_capture(self, enable: bool = True) -> None:
        """Runs device-batch passes as captured CUDA graphs (replayed while identical)."""
        _lib.check(self._lib.mp_engine_set_graph_capture(self.handle, 1 if enable else 0))

    def autotune_reset(self) -> None:
        """Restores the built-in kernel choice."""
        _lib.check(self._lib.mp_engine_autotune_reset(self.handle))

    def release_buffers(self) -> None:
        """Frees the device buffers kept between calls (mp_engine_release_buffers)."""
        db = getattr(self, "_one_shot", None)
        if db is not None:
            db.close()
            self._one_shot = None
        _lib.check(self._lib.mp_engine_release_buffers(self.handle))

    def fp32_peak_tflops(self) -> float:
        """Measured FP32 FMA throughput of this device (TFLOP/s)."""
        v = ctypes.c_double()
        _lib.check(self._lib.mp_measure_fp32_peak(self.handle, v))
        return float(v.value)

    def close(self) -> None:
        db = getattr(self, "_one_shot", None)
        if db is not None:
            db.close()
            self._one_shot = None
        if self.handle:
            self._lib.mp_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Model:
    """Forward- and reverse-strand machines resident on the device."""

    def __init__(self, engine: Engine, forward: StateModel, reverse: StateModel):
        self.engine = engine
        self._fd, self._rd = forward.desc(), reverse.desc()
        self._keep = (forward, reverse)
        h = c_void_p()
        _lib.check(engine._lib.mp_model_create(engine.handle, ctypes.byref(self._fd), ctypes.byref(self._rd),
                                               ctypes.byref(h)))
        self.handle = h

    @classmethod
    def from_polish(cls, engine: Engine, pm: PolishModel) -> "Model":
        return cls(engine, pm.forward, pm.reverse)

    def close(self) -> None:
        if self.handle:
            self.engine._lib.mp_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Jobs:
    """A batch of alignment jobs (host arrays). Job j aligns
    y_symbols[y_offsets[j]:y_offsets[j+1]] against x_symbols[x_begin[j]:x_end[j]]."""

    x_symbols: np.ndarray
    x_begin: np.ndarray
    x_end: np.ndarray
    y_symbols: np.ndarray
    y_offsets: np.ndarray
    anchors: np.ndarray          # (n, 3) int32 in job coordinates
    anchor_offsets: np.ndarray
    strand: np.ndarray           # uint8, 1 forward
    ragged_left: Optional[np.ndarray] = None
    ragged_right: Optional[np.ndarray] = None
    x_shift: Optional[np.ndarray] = None
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        self.x_symbols = np.ascontiguousarray(self.x_symbols, dtype=np.uint16)
        self.x_begin = np.ascontiguousarray(self.x_begin, dtype=np.int64)
        self.x_end = np.ascontiguousarray(self.x_end, dtype=np.int64)
        self.y_symbols = np.ascontiguousarray(self.y_symbols, dtype=np.uint16)
        self.y_offsets = np.ascontiguousarray(self.y_offsets, dtype=np.int64)
        self.anchors = np.ascontiguousarray(np.asarray(self.anchors, dtype=np.int32).reshape(-1, 3))
        self.anchor_offsets = np.ascontiguousarray(self.anchor_offsets, dtype=np.int64)
        self.strand = np.ascontiguousarray(self.strand, dtype=np.uint8)
        for name in ("ragged_left", "ragged_right"):
            v = getattr(self, name)
            if v is not None:
                setattr(self, name, np.ascontiguousarray(v, dtype=np.uint8))
        if self.x_shift is not None:
            self.x_shift = np.ascontiguousarray(self.x_shift, dtype=np.int64)

    @property
    def n_jobs(self) -> int:
        return int(self.x_begin.shape[0])

    def struct(self) -> _lib.Batch:
        b = _lib.Batch()
        b.n_jobs = self.n_jobs
        b.x_begin = _lib.ptr(self.x_begin, c_int64)
        b.x_end = _lib.ptr(self.x_end, c_int64)
        b.x_symbols_length = int(self.x_symbols.shape[0])
        xs = self.x_symbols if self.x_symbols.size else np.zeros(1, np.uint16)
        ys = self.y_symbols if self.y_symbols.size else np.zeros(1, np.uint16)
        an = self.anchors if self.anchors.size else np.zeros((1, 3), np.int32)
        self._keep = [xs, ys, an]
        b.x_symbols = _lib.ptr(xs, c_uint16)
        b.y_offsets = _lib.ptr(self.y_offsets, c_int64)
        b.y_symbols = _lib.ptr(ys, c_uint16)
        b.anchor_offsets = _lib.ptr(self.anchor_offsets, c_int64)
        b.anchors = _lib.ptr(an, c_int32)
        b.strand = _lib.ptr(self.strand, c_uint8)
        b.ragged_left = _lib.ptr(self.ragged_left, c_uint8)
        b.ragged_right = _lib.ptr(self.ragged_right, c_uint8)
        b.x_shift = _lib.ptr(self.x_shift, c_int64)
        return b

    @classmethod
    def single(cls, sx, sy, anchors, strand: int = 1, ragged_left: bool = False, ragged_right: bool = False,
               x_shift: int = 0) -> "Jobs":
        sx = np.asarray(sx, dtype=np.uint16)
        sy = np.asarray(sy, dtype=np.uint16)
        a = np.asarray(anchors, dtype=np.int32).reshape(-1, 3)
        return cls(sx, np.array([0]), np.array([sx.size]), sy, np.array([0, sy.size]), a,
                   np.array([0, a.shape[0]]), np.array([strand]), np.array([int(ragged_left)]),
                   np.array([int(ragged_right)]), np.array([x_shift]))

    @classmethod
    def concat(cls, parts: "list[Jobs]") -> "Jobs":
        """One batch holding the jobs of `parts` in order (templates are laid end to end)."""
        xs, xb, xe, ys, yo, an, ao, st, rl, rr, sh = [], [], [], [], [0], [], [0], [], [], [], []
        x_base = 0
        for p in parts:
            n = p.n_jobs
            xs.append(p.x_symbols)
            xb.append(p.x_begin + x_base)
            xe.append(p.x_end + x_base)
            x_base += p.x_symbols.size
            ys.append(p.y_symbols)
            yo.extend((p.y_offsets[1:] + yo[-1]).tolist())
            an.append(p.anchors)
            ao.extend((p.anchor_offsets[1:] + ao[-1]).tolist())
            st.append(p.strand)
            rl.append(p.ragged_left if p.ragged_left is not None else np.zeros(n, np.uint8))
            rr.append(p.ragged_right if p.ragged_right is not None else np.zeros(n, np.uint8))
            sh.append(p.x_shift if p.x_shift is not None else np.zeros(n, np.int64))

        def cat(v, dt):
            return np.concatenate(v).astype(dt) if v else np.zeros(0, dt)

        return cls(cat(xs, np.uint16), cat(xb, np.int64), cat(xe, np.int64), cat(ys, np.uint16),
                   np.asarray(yo, np.int64), np.concatenate(an) if an else np.zeros((0, 3), np.int32),
                   np.asarray(ao, np.int64), cat(st, np.uint8), cat(rl, np.uint8), cat(rr, np.uint8),
                   cat(sh, np.int64))


@dataclass
class Pairs:
    """Posterior tuples of a batch: for list k (0 match, 1 gap-x, 2 gap-y), job j owns
    rows offsets[k][j]:offsets[k][j+1] of weight/x/y."""

    offsets: list
    weight: list
    x: list
    y: list
    log_likelihood: np.ndarray
    cells: np.ndarray
    total_cells: int
    device_ms: float

    def job(self, j: int, k: int) -> np.ndarray:
        a, b = self.offsets[k][j], self.offsets[k][j + 1]
        return np.stack([self.weight[k][a:b], self.x[k][a:b], self.y[k][a:b]], axis=1)


def _copy_view(lib, res) -> Pairs:
    v = _lib.ResultView()
    _lib.check(lib.mp_result_view_get(res, ctypes.byref(v)))
    n = v.n_jobs
    offsets, w, x, y = [], [], [], []
    for k in range(3):
        off = np.ctypeslib.as_array(v.offsets[k], shape=(n + 1,)).copy() if n >= 0 else np.zeros(1, np.int64)
        tot = int(off[-1]) if n > 0 else 0
        offsets.append(off)
        for dst, src in ((w, v.weight[k]), (x, v.x[k]), (y, v.y[k])):
            dst.append(np.ctypeslib.as_array(src, shape=(tot,)).copy() if tot else np.zeros(0, np.int32))
    ll = np.ctypeslib.as_array(v.log_likelihood, shape=(n,)).copy() if n else np.zeros(0)
    cells = np.ctypeslib.as_array(v.cells, shape=(n,)).copy() if n else np.zeros(0, np.int64)
    return Pairs(offsets, w, x, y, ll, cells, int(v.total_cells), float(v.device_ms))


def pinned_empty(shape, dtype) -> np.ndarray:
    """An uninitialised numpy array in page-locked host memory (freed with the array); copies
    between it and the device run by DMA at full link speed."""
    lib = _lib.load()
    dtype = np.dtype(dtype)
    n = int(np.prod(shape)) * dtype.itemsize
    p = c_void_p()
    _lib.check(lib.mp_host_alloc(max(n, 1), ctypes.byref(p)))
    buf = (ctypes.c_char * max(n, 1)).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)
    weakref.finalize(buf, lib.mp_host_free, c_void_p(p.value))
    return arr


class OutputBuffer:
    """Reusable host arrays for the results of batches (page-locked by default). A call that
    writes into the buffer returns Pairs whose arrays are views of it, valid until the buffer
    is used again."""

    def __init__(self, pinned: bool = True):
        self.pinned = pinned
        self._tuples = [None, None, None]  # per list: (3, capacity) int32 rows weight, x, y
        self._jobs = None                  # (offsets (3, n+1) int64, log_likelihood (n,), cells (n,))
        self._n = -1

    def _alloc(self, shape, dtype):
        return pinned_empty(shape, dtype) if self.pinned else np.empty(shape, dtype)

    def ensure(self, n_jobs: int, totals) -> None:
        if self._n < n_jobs:
            cap = max(n_jobs, int(self._n * 1.25) if self._n > 0 else 0)
            self._jobs = (self._alloc((3, cap + 1), np.int64), self._alloc((cap,), np.float64),
                          self._alloc((cap,), np.int64))
            self._n = cap
        for k in range(3):
            need = int(totals[k])
            t = self._tuples[k]
            if t is None or t.shape[1] < need:
                self._tuples[k] = self._alloc((3, max(need + need // 8, 1)), np.int32)

    def struct(self) -> "_lib.Output":
        o = _lib.Output()
        offs, ll, cells = self._jobs
        for k in range(3):
            o.offsets[k] = _lib.ptr(offs[k], c_int64)
            t = self._tuples[k]
            o.weight[k] = _lib.ptr(t[0], c_int32)
            o.x[k] = _lib.ptr(t[1], c_int32)
            o.y[k] = _lib.ptr(t[2], c_int32)
        o.log_likelihood = _lib.ptr(ll, ctypes.c_double)
        o.cells = _lib.ptr(cells, c_int64)
        return o

    def pairs(self, n_jobs: int, totals, device_ms: float) -> Pairs:
        offs, ll, cells = self._jobs
        offsets = [offs[k, :n_jobs + 1] for k in range(3)]
        w = [self._tuples[k][0, :int(totals[k])] for k in range(3)]
        x = [self._tuples[k][1, :int(totals[k])] for k in range(3)]
        y = [self._tuples[k][2, :int(totals[k])] for k in range(3)]
        c = cells[:n_jobs]
        return Pairs(offsets, w, x, y, ll[:n_jobs], c, int(c.sum()), device_ms)


def realign_batch(engine: Engine, model: Model, params: AlignmentParams, jobs: Jobs,
                  out: Optional[OutputBuffer] = None) -> Pairs:
    """Full posterior pass over a batch held in host memory (H2D, kernels, D2H inside).

    The engine keeps the device batch of its last call and reuses its buffers. Results go into
    `out` when given (views valid until `out` is reused), else into new numpy arrays."""
    db = getattr(engine, "_one_shot", None)
    if db is None or db.model is not model:
        if db is not None:
            db.close()
        db = DeviceBatch(engine, model, params, jobs)
        engine._one_shot = db
    else:
        db.reset(jobs, params)
    ms = db.run()
    return db.fetch_into(out if out is not None else OutputBuffer(pinned=False), ms)


def realign_batch_pipelined(engine: Engine, model: Model, params: AlignmentParams, jobs: Jobs,
                            out: Optional[OutputBuffer] = None, parts: int = 0) -> Pairs:
    """The same pass as realign_batch, pipelined (mp_realign_batch_into): slices of the jobs
    alternate between two streams so that one slice's copies overlap another's kernels. Results
    go into `out` (page-locked by default; grown and the call repeated when a list does not
    fit) and are returned as views of it."""
    out = out if out is not None else OutputBuffer(pinned=True)
    n = jobs.n_jobs
    lib = engine._lib
    ps, bs = params.struct(), jobs.struct()
    out.ensure(n, [t.shape[1] if t is not None else 0 for t in out._tuples])
    need = (c_int64 * 3)()
    for attempt in range(2):
        o = out.struct()
        cap = (c_int64 * 3)(*[out._tuples[k].shape[1] for k in range(3)])
        st = lib.mp_realign_batch_into(engine.handle, model.handle, ctypes.byref(ps), ctypes.byref(bs), int(parts),
                                       ctypes.byref(o), cap, need)
        if st == _lib.MP_ERR_OVERFLOW and attempt == 0:
            out.ensure(n, [int(need[k]) for k in range(3)])
            continue
        _lib.check(st)
        break
    return out.pairs(n, [int(need[k]) for k in range(3)], 0.0)


class DeviceBatch:
    """A batch resident in HBM; ``run`` times only the device work (band + posterior kernels)."""

    def __init__(self, engine: Engine, model: Model, params: AlignmentParams, jobs: Jobs):
        self.engine, self.model, self.params, self.jobs = engine, model, params, jobs
        self._ps = params.struct()
        self._bs = jobs.struct()
        h = c_void_p()
        _lib.check(engine._lib.mp_device_batch_create(engine.handle, model.handle, ctypes.byref(self._ps),
                                                      ctypes.byref(self._bs), ctypes.byref(h)))
        self.handle = h

    def run(self) -> float:
        ms = c_float(0.0)
        _lib.check(self.engine._lib.mp_device_batch_run(self.engine.handle, self.handle, ctypes.byref(ms)))
        return float(ms.value)

    def fetch(self) -> Pairs:
        lib = self.engine._lib
        res = c_void_p()
        _lib.check(lib.mp_device_batch_fetch(self.engine.handle, self.handle, ctypes.byref(res)))
        try:
            return _copy_view(lib, res)
        finally:
            lib.mp_result_destroy(res)

    def reset(self, jobs: Jobs, params: Optional[AlignmentParams] = None) -> None:
        """Replaces the jobs (and parameters), reusing the batch's device buffers."""
        if params is not None:
            self.params = params
            self._ps = params.struct()
        self.jobs = jobs
        self._bs = jobs.struct()
        _lib.check(self.engine._lib.mp_device_batch_reset(self.engine.handle, self.handle, ctypes.byref(self._ps),
                                                          ctypes.byref(self._bs)))

    def run_plain(self, max_tasks: int):
        """The plain form: one launch of one warp per sub-problem for the first `max_tasks`
        sub-problems. Returns (posterior-kernel ms, cells run)."""
        ms, cells = c_float(0.0), c_int64(0)
        _lib.check(self.engine._lib.mp_device_batch_run_plain(self.engine.handle, self.handle, int(max_tasks),
                                                              ctypes.byref(ms), ctypes.byref(cells)))
        return float(ms.value), int(cells.value)

    def counts(self):
        t = (c_int64 * 3)()
        _lib.check(self.engine._lib.mp_device_batch_counts(self.handle, t))
        return [int(t[0]), int(t[1]), int(t[2])]

    def fetch_into(self, out: OutputBuffer, device_ms: float = 0.0) -> Pairs:
        """Copies the last run's results into `out` (no host allocation when it is large
        enough) and returns them as views of it."""
        totals = self.counts()
        n = self.jobs.n_jobs
        out.ensure(n, totals)
        o = out.struct()
        _lib.check(self.engine._lib.mp_device_batch_fetch_into(self.engine.handle, self.handle, ctypes.byref(o)))
        return out.pairs(n, totals, device_ms)

    def timing(self):
        """(band_ms, posterior_ms) CUDA-event times of the last run."""
        b, q = c_float(), c_float()
        _lib.check(self.engine._lib.mp_device_batch_timing(self.handle, b, q))
        return float(b.value), float(q.value)

    def stats(self):
        cells, tasks, launches = c_int64(), c_int64(), ctypes.c_int32()
        _lib.check(self.engine._lib.mp_device_batch_stats(self.handle, cells, tasks, launches))
        return cells.value, tasks.value, launches.value

    def close(self) -> None:
        if self.handle:
            self.engine._lib.mp_device_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def get_aligned_pairs_with_indels_using_anchors(engine: Engine, model: Model, sx, sy, anchors,
                                                params: AlignmentParams, strand: int = 1,
                                                ragged_left: bool = False, ragged_right: bool = False):
    """(matches, gap_x, gap_y) as (n, 3) int arrays of (weight, x, y) for one read."""
    r = realign_batch(engine, model, params, Jobs.single(sx, sy, anchors, strand, ragged_left, ragged_right))
    return r.job(0, 0), r.job(0, 1), r.job(0, 2)


def get_aligned_pairs_using_anchors(engine: Engine, model: Model, sx, sy, anchors, params: AlignmentParams,
                                    strand: int = 1, ragged_left: bool = False, ragged_right: bool = False):
    return get_aligned_pairs_with_indels_using_anchors(engine, model, sx, sy, anchors, params, strand,
                                                       ragged_left, ragged_right)[0]


def forward_batch(engine: Engine, model: Model, params: AlignmentParams, jobs: Jobs) -> np.ndarray:
    """ln P of every job over the band of band_construct (fixed expansion
    params.diagonal_expansion; the anchors' own expansions are ignored), no splits."""
    out = np.zeros(max(jobs.n_jobs, 1), dtype=np.float64)
    ps, bs = params.struct(), jobs.struct()
    _lib.check(engine._lib.mp_forward_batch(engine.handle, model.handle, ctypes.byref(ps), ctypes.byref(bs),
                                            _lib.ptr(out, ctypes.c_double)))
    return out[:jobs.n_jobs]


def compute_forward_probability(engine: Engine, model: Model, sx, sy, anchors, params: AlignmentParams,
                                strand: int = 1, ragged_left: bool = False, ragged_right: bool = False) -> float:
    """computeForwardProbability for one pair of sequences (anchors may be empty)."""
    return float(forward_batch(engine, model, params, Jobs.single(sx, sy, anchors, strand, ragged_left,
                                                                  ragged_right))[0])


def forward_pairs(engine: Engine, model: Model, x_symbols, y_symbols, x_offset, x_length, y_offset, y_length,
                  strand) -> np.ndarray:
    """computeForwardProbability without anchors for many (allele, read substring) pairs, as
    the bubble graph calls it (impl/bubbleGraph.c:924), in the reference's arithmetic (see
    mp_forward_pairs): pair j aligns x_symbols[x_offset[j]:+x_length[j]] against
    y_symbols[y_offset[j]:+y_length[j]] with the forward (strand 1) or reverse model."""
    xs = np.ascontiguousarray(x_symbols, dtype=np.uint16)
    ys = np.ascontiguousarray(y_symbols, dtype=np.uint16)
    xo = np.ascontiguousarray(x_offset, dtype=np.int64)
    xl = np.ascontiguousarray(x_length, dtype=np.int32)
    yo = np.ascontiguousarray(y_offset, dtype=np.int64)
    yl = np.ascontiguousarray(y_length, dtype=np.int32)
    st = np.ascontiguousarray(strand, dtype=np.uint8)
    n = xo.size
    if not (xl.size == yo.size == yl.size == st.size == n):
        raise ValueError("one offset, length and strand per pair")
    b = _lib.PairBatch(n, _lib.ptr(xo, ctypes.c_int64), _lib.ptr(xl, ctypes.c_int32), _lib.ptr(yo, ctypes.c_int64),
                       _lib.ptr(yl, ctypes.c_int32), _lib.ptr(st, ctypes.c_uint8), xs.size,
                       _lib.ptr(xs if xs.size else np.zeros(1, np.uint16), ctypes.c_uint16), ys.size,
                       _lib.ptr(ys if ys.size else np.zeros(1, np.uint16), ctypes.c_uint16))
    out = np.zeros(max(n, 1), dtype=np.float64)
    _lib.check(engine._lib.mp_forward_pairs(engine.handle, model.handle, ctypes.byref(b), _lib.ptr(out, ctypes.c_double)))
    return out[:n]


def match_pairs_reference(engine: Engine, model: Model, params: AlignmentParams, jobs: "Jobs") -> List[np.ndarray]:
    """getAlignedPairs of anchor-free jobs in the reference's own arithmetic (see
    mp_match_pairs_reference): per job an (n, 3) array of (weight, x, y) in the reference's
    order. The model must be without run lengths (the code-default nucleotide machine)."""
    ps, bs = params.struct(), jobs.struct()
    offs = np.zeros(jobs.n_jobs + 1, np.int64)
    total = ctypes.c_int64(0)
    cap = int(sum((jobs.x_end[j] - jobs.x_begin[j]) * (jobs.y_offsets[j + 1] - jobs.y_offsets[j])
                  for j in range(jobs.n_jobs))) + 1
    w, x, y = (np.zeros(cap, np.int32) for _ in range(3))
    _lib.check(engine._lib.mp_match_pairs_reference(engine.handle, model.handle, ctypes.byref(ps), ctypes.byref(bs),
                                                    _lib.ptr(offs, ctypes.c_int64), _lib.ptr(w, ctypes.c_int32),
                                                    _lib.ptr(x, ctypes.c_int32), _lib.ptr(y, ctypes.c_int32), cap,
                                                    ctypes.byref(total)))
    return [np.stack([w[offs[j]:offs[j + 1]], x[offs[j]:offs[j + 1]], y[offs[j]:offs[j + 1]]], axis=1).astype(np.int64)
            for j in range(jobs.n_jobs)]


def forward_pairs_timing(engine: Engine) -> dict:
    """The last forward_pairs call: kernel_ms (device time of its launches), cells, pairs."""
    ms = ctypes.c_float(0.0)
    cells = ctypes.c_int64(0)
    pairs = ctypes.c_int64(0)
    _lib.check(engine._lib.mp_forward_pairs_timing(engine.handle, ctypes.byref(ms), ctypes.byref(cells),
                                                   ctypes.byref(pairs)))
    return {"kernel_ms": ms.value, "cells": cells.value, "pairs": pairs.value}


@dataclass
class Expectations:
    """Expected counts of a batch (see mp_expectations_batch): per model m (0 forward
    strand, 1 reverse) transitions[m] (3x3, from x to), match[m] (5x5, x base x y base),
    gap_x[m], gap_y[m] (5), start[m], end[m] (state posteriors at the first / last cell),
    repeat[t] (4 x 51 x 51 by run-length table), the summed ln P and each job's ln P."""
    transitions: np.ndarray
    match: np.ndarray
    gap_x: np.ndarray
    gap_y: np.ndarray
    start: np.ndarray
    end: np.ndarray
    repeat: np.ndarray
    log_likelihood: float
    job_log_likelihood: np.ndarray


def expectations_batch(engine: Engine, model: Model, params: AlignmentParams, jobs: Jobs) -> Expectations:
    """Gradient of the summed log-likelihood with respect to the log transition and
    emission parameters (expected counts), from the adjoint kernel."""
    e = _lib.Expectations()
    ll = np.zeros(max(jobs.n_jobs, 1), dtype=np.float64)
    ps, bs = params.struct(), jobs.struct()
    _lib.check(engine._lib.mp_expectations_batch(engine.handle, model.handle, ctypes.byref(ps), ctypes.byref(bs),
                                                 ctypes.byref(e), _lib.ptr(ll, ctypes.c_double)))
    arr = lambda v, shape: np.ctypeslib.as_array(v).reshape(shape).copy()  # noqa: E731
    return Expectations(arr(e.transitions, (2, 3, 3)), arr(e.match, (2, 5, 5)), arr(e.gap_x, (2, 5)),
                        arr(e.gap_y, (2, 5)), arr(e.start, (2, 3)), arr(e.end, (2, 3)),
                        arr(e.repeat, (2, 4, 51, 51)), float(e.log_likelihood),
                        ll[:jobs.n_jobs].copy())
