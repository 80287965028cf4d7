#!/usr/bin/env python3
"""Throughput of the banded pair-HMM forward/backward/posterior pass (GCUPS) on B200.

Workload (default): the batched uneven-reads configuration -- 256 chunks of a
10 kb homopolymer-enriched synthetic template (GC 0.41, run lengths geometric
p=0.55 capped at 20), 30x coverage, log-normal read lengths (median 6 kb,
sigma 0.6) truncated to the chunk, nanopore-like errors, band half-width 25,
the shipped run-length model; all reads of all chunks in one persistent launch.
A step is one full posterior pass over the batch. Cells = sum of anti-diagonal
band widths (the reference's band). Inputs are larger than L2 (126 MB).

value: cells / device time (band + posterior kernels, CUDA events) with inputs
resident in HBM. e2e: the same pass through mp_realign_batch_into (pipelined) with host
buffers in pinned memory (host->device copies, planning, kernels, compaction
and device->host copies of every tuple inside the timed region).

--impl reference: the reference's own C implementation (pairwiseAligner.c /
stateMachine.c compiled unmodified) on all host cores, OpenMP over chunks with
schedule(dynamic,1) and the reads of a chunk in order (marginPolish.c:436-439),
timed on a prefix of whole chunks of the same workload; its cells come from the
reference's own band construction. That arm loads no library of this package:
the workload generator is numpy only.

Multi-GPU: one process per GPU (torchrun); reads are independent, so every rank
runs its own full workload (weak scaling, no data-path collective); value is
the sum of cells over ranks divided by the max device time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOP_PER_CELL = 48  # 30 FP32 FMA-pipe instructions per cell (forward 12, backward 12, posterior 6)
# DRAM bytes (read + write) per band cell of the posterior kernel, from one ncu capture of the
# same kernel on a 24-chunk slice of the workload; traffic grows with cells, so a full launch
# moves this times its cells.
DRAM_BYTES_PER_CELL = 6.08
METRIC = "GCUPS fwd+bwd+posterior (batched FP32 vs plain GPU, ≤1e-4 vs FP64); CPU ref"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["batched", "small"], default="batched")
    ap.add_argument("--chunks", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=8.0, help="CPU work per baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--plain-reads", type=int, default=96, help="reads timed in the plain one-read-per-launch form")
    ap.add_argument("--lanes", type=int, default=0, choices=[0, 8, 16, 32],
                    help="lanes per banded sub-problem (0 = the engine's automatic choice)")
    ap.add_argument("--warps", type=int, default=0, help="warps per block of the posterior kernel (0 = automatic)")
    ap.add_argument("--no-graphs", action="store_true", help="direct launches instead of CUDA graph replay")
    ap.add_argument("--autotune-chunks", type=int, default=24,
                    help="chunks of the separate seeded sample the autotuner times the kernel variants on (0 = off)")
    ap.add_argument("--chunks-5mb", type=int, default=50,
                    help="chunks of the 5 Mb configuration (of 50) whose realignment pass is measured")
    ap.add_argument("--no-scale", action="store_true",
                    help="skip the 1 Mb polishing-loop and 5 Mb realignment-pass measurements")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the adjoint and POA-loop measurements reported beside the headline")
    ap.add_argument("--bubble-scores", action="store_true",
                    help="only the polish step's bubble-score measurement (one JSON line; no CPU sample)")
    ap.add_argument("--polish-shipped", action="store_true",
                    help="only the shipped polishing loop's measurement, with its per-step times (one JSON line)")
    ap.add_argument("--device-indels", action="store_true",
                    help="the shipped loop finds the reads' indel candidates on the GPU (the default)")
    ap.add_argument("--host-indels", action="store_true",
                    help="the shipped loop finds the reads' indel candidates on the host threads")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            if len(s) < 9:
                continue
            for i, n in enumerate(names):
                if s[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def load_model():
    from marginpolish_b200 import params
    return params.polish_model_from_npz(os.path.join(ROOT, "tests", "golden", "model_np.npz"))


def make_workload(args, rank):
    from marginpolish_b200 import synth
    if args.config == "small":
        return synth.config_small(seed=args.seed + rank)
    return synth.config_batched(seed=args.seed + rank, n_chunks=args.chunks)


def chunk_offsets(wl):
    """Job offsets of the workload's chunks (the jobs of a chunk are consecutive)."""
    import numpy as np
    t = np.asarray(wl.read_template, dtype=np.int64)
    assert t.size == 0 or np.all(np.diff(t) >= 0)
    off = np.zeros(len(wl.templates) + 1, dtype=np.int64)
    off[1:] = np.cumsum(np.bincount(t, minlength=len(wl.templates)))
    return off


def job_prefix(jobs, n):
    """The first n jobs of a batch."""
    from marginpolish_b200 import Jobs
    a0, a1 = int(jobs.anchor_offsets[0]), int(jobs.anchor_offsets[n])
    return Jobs(jobs.x_symbols, jobs.x_begin[:n], jobs.x_end[:n], jobs.y_symbols[:int(jobs.y_offsets[n])],
                jobs.y_offsets[:n + 1], jobs.anchors[a0:a1], jobs.anchor_offsets[:n + 1], jobs.strand[:n])


def reference_models(ref, pm):
    import numpy as np
    z = np.load(os.path.join(ROOT, "tests", "golden", "model_np.npz"))
    hf = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    return hf, hr


def reference_cells(ref, jobs, pm):
    """Cells per job from the reference's own band construction (band_constructDynamic,
    impl/pairwiseAligner.c:120-173, run through Oracle A)."""
    import numpy as np
    ap = pm.alignment
    out = np.zeros(jobs.n_jobs, dtype=np.int64)
    for j in range(jobs.n_jobs):
        lx = int(jobs.x_end[j] - jobs.x_begin[j])
        ly = int(jobs.y_offsets[j + 1] - jobs.y_offsets[j])
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        out[j] = ref.band_cells(a, lx, ly, ap.diagonal_expansion, ap.dynamic_anchor_expansion)
    return out


class ReferenceCpu:
    """Oracle A (the reference's own code) on whole chunks: OpenMP over chunks with
    schedule(dynamic,1) on all host cores, each chunk's reads in order on one thread."""

    def __init__(self, pm, jobs, offsets):
        from oracle.bindings import RefOracle
        self.ref = RefOracle()
        self.pm = pm
        self.jobs = jobs
        self.offsets = offsets
        self.hf, self.hr = reference_models(self.ref, pm)
        self.cores = os.cpu_count() or 1

    def sample(self, n_chunks):
        n_chunks = max(1, min(n_chunks, self.offsets.size - 1))
        sub = job_prefix(self.jobs, int(self.offsets[n_chunks]))
        return sub, self.offsets[:n_chunks + 1], int(reference_cells(self.ref, sub, self.pm).sum())

    def run(self, sample, threads):
        sub, off, _ = sample
        t = time.perf_counter()
        self.ref.align_chunks(self.hf, self.hr, sub, off, self.pm.alignment, threads)
        return time.perf_counter() - t

    def calibrated_sample(self, seconds):
        """A prefix of whole chunks, a multiple of the core count, of about `seconds` of work."""
        probe = self.sample(self.cores)
        t = self.run(probe, self.cores)
        rounds = max(1, int(round(seconds / max(t, 1e-3))))
        return probe if rounds == 1 else self.sample(self.cores * rounds)

    def close(self):
        self.ref.free_model(self.hf)
        self.ref.free_model(self.hr)


def time_reference(pm, wl, jobs, seconds, steps=1, warmup=0):
    """The reference's CPU rate (GCUPS) on a prefix of whole chunks, all cores, plus one core on
    the first chunk."""
    import numpy as np
    rc = ReferenceCpu(pm, jobs, chunk_offsets(wl))
    sample = rc.calibrated_sample(seconds)
    for _ in range(warmup):
        rc.run(sample, rc.cores)
    times = [rc.run(sample, rc.cores) for _ in range(steps)]
    one = rc.sample(1)
    t1 = rc.run(one, 1)
    rc.close()
    n_chunks = sample[1].size - 1
    return {"gcups": sample[2] / float(np.median(times)) / 1e9, "cores": rc.cores, "chunks": n_chunks,
            "reads": int(sample[1][-1]), "cells": sample[2], "seconds": float(np.median(times)),
            "gcups_1core": one[2] / max(t1, 1e-9) / 1e9, "reads_1core": int(one[1][-1])}


def accuracy_sample(jobs, res, pm, n_reads=6):
    """The timed batch's results on its first reads against the exact FP64 oracle (the checker,
    run in the CPU-baseline leg): max |posterior - FP64| over every emitted tuple, and the
    relative log-likelihood error."""
    from oracle.bindings import ExactOracle, MpoModel
    from oracle.compare import check_job
    eo = ExactOracle()
    models = (MpoModel.from_state_model(pm.forward), MpoModel.from_state_model(pm.reverse))
    worst, worst_ll, tuples = 0.0, 0.0, 0
    n = min(n_reads, jobs.n_jobs)
    for j in range(n):
        sx = jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]]
        sy = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        o = eo.align_with_indels(models[0] if jobs.strand[j] else models[1], sx, sy, a, pm.alignment, dense=True)
        g = [res.job(j, k).copy() for k in range(3)]
        shift = int(jobs.x_shift[j]) if jobs.x_shift is not None else 0
        for k in range(3):
            g[k][:, 1] -= shift
            tuples += g[k].shape[0]
        worst = max(worst, check_job(g, o, pm.alignment.threshold)["max_abs_posterior_error"])
        ll = o["log_likelihood"]
        worst_ll = max(worst_ll, abs(float(res.log_likelihood[j]) - ll) / max(1.0, abs(ll)))
    return {"reads": n, "tuples": tuples, "max_abs_posterior_error_vs_fp64": worst,
            "max_rel_loglik_error_vs_fp64": worst_ll, "bar": "posteriors 1e-4 absolute, log-likelihood 1e-5 relative"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    from oracle.bindings import available_reference
    if not available_reference():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libref_oracle.so missing"}))
        return
    pm = load_model()
    wl = make_workload(args, 0)
    jobs = wl.jobs()
    r = time_reference(pm, wl, jobs, args.cpu_seconds, steps=args.steps, warmup=args.warmup)
    sample = (f"rate on a prefix of {r['chunks']} whole chunks ({r['reads']} reads, {r['cells']} cells) of the "
              f"{len(wl.templates)}-chunk workload per step, OpenMP over chunks (schedule(dynamic,1)) on "
              f"{r['cores']} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": r["gcups"], "unit": "GCUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["seconds"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"{args.config}: {wl.meta}", "sample": sample, "chunks_in_sample": r["chunks"],
                   "reads_in_sample": r["reads"], "cells_per_step": r["cells"]},
        "cpu_baseline": {"value": r["gcups"], "unit": "GCUPS", "cores": r["cores"], "kind": "reference",
                         "sample": sample, "value_1core": r["gcups_1core"],
                         "sample_1core": f"first chunk ({r['reads_1core']} reads), 1 thread"},
        "e2e": {"value": r["gcups"], "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def band_cells(jobs, pm):
    """Cells per job from the library's host band restatement (integer-exact)."""
    import ctypes

    import numpy as np
    from marginpolish_b200 import _lib
    lib = _lib.load()
    out = np.zeros(jobs.n_jobs, dtype=np.int64)
    ap = pm.alignment
    for j in range(jobs.n_jobs):
        lx = int(jobs.x_end[j] - jobs.x_begin[j])
        ly = int(jobs.y_offsets[j + 1] - jobs.y_offsets[j])
        a = np.ascontiguousarray(jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]])
        b = np.zeros((lx + ly + 1, 3), dtype=np.int64)
        _lib.check(lib.mp_band(_lib.ptr(a, ctypes.c_int32) if a.size else None, a.shape[0], lx, ly,
                               ap.diagonal_expansion, 1 if ap.dynamic_anchor_expansion else 0,
                               _lib.ptr(b, ctypes.c_int64)))
        out[j] = int(((b[:, 2] - b[:, 1]) // 2 + 1).sum()) if lx + ly > 0 else 0
    return out


def measure_adjoint(engine, model, pm):
    """The adjoint (expected counts) over the gradient workload: 512 reads of 2-5 kb on 64
    random 5 kb templates; one call of mp_expectations_batch (host arrays in, counts out)."""
    import numpy as np
    from marginpolish_b200 import expectations_batch, synth
    wl = synth.config_adjoint(seed=4)
    jobs = wl.jobs()
    cells = int(band_cells(jobs, pm).sum())
    expectations_batch(engine, model, pm.alignment, jobs)  # warm
    ts = []
    for _ in range(3):
        t = time.perf_counter()
        ex = expectations_batch(engine, model, pm.alignment, jobs)
        ts.append(time.perf_counter() - t)
    t = float(np.median(ts))
    return {"workload": "512 reads of 2-5 kb on 64 random 5 kb templates, band half-width 25", "reads": jobs.n_jobs,
            "cells": cells, "seconds": t, "gcups": cells / t / 1e9, "log_likelihood": ex.log_likelihood,
            "form": "mp_expectations_batch, host arrays in / counts out (FP32 cells, FP64 accumulation)"}


# FP64 adds and products of one cell of the bubble scorer with a switch-free model: three
# incoming terms f + (e + t) of the match state, two of each gap state (2 operations each), the
# run-length emission sum, and four approximate log-sums (a subtraction, a three-step cubic and
# the final addition: 8 each)
DP_OPS_PER_PAIR_CELL = 14 + 1 + 32


def polish_workload():
    """8 chunks of a homopolymer-enriched 10 kb template at 50x, reads of 3-9 kb with seeded
    nanopore-like base qualities, drafts with 1% homopolymer-biased indels."""
    from marginpolish_b200 import synth
    wl = synth.config_polish(seed=41, n_chunks=8, chunk_len=10_000, coverage=50, read_len=(3000, 9000), hp_runs=True)
    return wl, wl.qualities(41)


def measure_bubble_scoring(engine, model, pm, cpu_sample=True):
    """The scoring step of the polish step's bubble graphs (impl/bubbleGraph.c:905-955) on real
    graphs: the first realignment of the polish workload, every chunk's bubble graph, then one
    mp_forward_pairs launch over every (allele, distinct read substring) pair of every bubble,
    in the reference's arithmetic (FP64 log cells, its approximate log-sum). The reference's own
    bubbleGraph_constructFromPoa, which computes the same scores one pair at a time, is timed
    on a sample chunk on one core."""
    import ctypes

    import numpy as np
    from marginpolish_b200 import PoaSet, PolishParams, _lib, forward_pairs_timing
    wl, quals = polish_workload()
    s = PoaSet.from_polish_model(engine, model, pm, PolishParams.shipped(), wl.drafts, wl.reads, wl.strands,
                                 wl.anchors, quals)
    s.realign()
    t = time.perf_counter()
    s.build_bubbles()
    build_s = time.perf_counter() - t
    s.score_bubbles()  # warm
    calls, kernels = [], []
    for _ in range(5):
        t = time.perf_counter()
        s.score_bubbles()
        calls.append(time.perf_counter() - t)
        kernels.append(forward_pairs_timing(engine)["kernel_ms"])
    tm = forward_pairs_timing(engine)
    n_bubbles = sum(len(s.bubbles(c)) for c in range(s.n_chunks))
    s.close()
    g = ctypes.c_double(0.0)
    _lib.check(engine._lib.mp_measure_fp64_peak(engine.handle, ctypes.byref(g)))
    k_ms = float(np.median(kernels))
    call_s = float(np.median(calls))
    achieved = tm["cells"] * DP_OPS_PER_PAIR_CELL / (k_ms * 1e-3) / 1e9
    out = {"workload": "bubble graphs of 8 chunks x 10 kb (homopolymer-enriched), 50x, reads of 3-9 kb with base "
                       "qualities, drafts with 1% homopolymer-biased indels",
           "bubbles": n_bubbles, "pairs": tm["pairs"], "cells": tm["cells"], "kernel_ms": k_ms,
           "call_ms": call_s * 1e3, "gcups_kernel": tm["cells"] / (k_ms * 1e-3) / 1e9,
           "gcups_call": tm["cells"] / call_s / 1e9, "pairs_per_s": tm["pairs"] / call_s,
           "build_ms": build_s * 1e3,
           "roofline": {"bound": "fp64", "achieved": achieved, "peak": g.value, "unit": "G FP64 ops/s",
                        "frac": achieved / g.value,
                        "note": f"{DP_OPS_PER_PAIR_CELL} FP64 adds/products per cell x cells / kernel event time; "
                                "peak = FP64 add/product issue rate measured live (mp_measure_fp64_peak)"},
           "form": "mp_poa_set_score_bubbles -> mp_forward_pairs: one thread per pair, reference arithmetic, "
                   "bit-identical scores"}
    if cpu_sample:
        out["cpu_reference"] = reference_bubble_sample(pm)
    return out


def reference_bubble_sample(pm):
    """The reference's bubbleGraph_constructFromPoa (oracle/_ref/libref_poa.so, one core) on the
    graph of one 3 kb chunk at 50x: seconds, and its rate over the pairs it scores."""
    import os as _os

    import numpy as np
    from marginpolish_b200 import PolishParams, synth
    from oracle.bindings import RefPoaOracle, available_reference_poa
    if not available_reference_poa():
        return {"unavailable": "reference POA build (oracle/_ref/libref_poa.so) not present"}
    ref = RefPoaOracle()
    z = np.load(_os.path.join(ROOT, "tests", "golden", "model_np.npz"))
    hf = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], False, z["repeat_log10"], 1)
    hr = ref.model(int(z["hmm_type"]), z["transitions"], z["emissions"], True, z["repeat_log10"], 0)
    wl = synth.config_polish(seed=9, n_chunks=1, chunk_len=3000, coverage=50, read_len=(1500, 2500), hp_runs=True)
    quals = wl.qualities(9)
    pp = PolishParams.shipped()
    params_h = ref.params(hf, hr, pm.alignment, max_iterations=0)
    ref.set_polish(params_h, pp)
    reads_h = ref.reads(wl.reads[0], wl.strands[0])
    ref.set_qualities(reads_h, quals[0])
    anchors_h = ref.anchors(wl.anchors[0])
    poa = ref.realign(reads_h, anchors_h, wl.drafts[0], params_h)
    t = time.perf_counter()
    g = ref.bubble_graph(poa, reads_h, params_h)
    sec = time.perf_counter() - t
    cells = pairs = 0
    for b in g["bubbles"]:
        seen = set()
        for read, start, length in b["reads"].tolist():
            r = wl.reads[0][read]
            key = (r.chars[start:start + length], tuple(int(v) for v in r.counts[start:start + length]))
            if key in seen:
                continue
            seen.add(key)
            for chars, _ in b["alleles"]:
                cells += (len(chars) + 1) * (length + 1)
                pairs += 1
    ref.free_poa(poa)
    ref.free_anchors(anchors_h)
    ref.free_reads(reads_h)
    ref.free_params(params_h)
    ref.free_model(hf)
    ref.free_model(hr)
    return {"seconds": sec, "bubbles": len(g["bubbles"]), "pairs": pairs, "cells": cells,
            "gcups": cells / sec / 1e9, "cores": 1, "kind": "reference",
            "sample": "bubbleGraph_constructFromPoa (construction and scores) on one 3 kb chunk at 50x, one core"}


def measure_polish_shipped(engine, model, pm, device_indels=True):
    """The shipped loop (poa_realignAll with one polish iteration, then the run-length estimate)
    over the polish workload: realignment, bubble graphs, scores, new consensus, anchors,
    second realignment."""
    from marginpolish_b200 import PoaSet, PolishParams
    wl, quals = polish_workload()
    best = None
    for _ in range(2):
        s = PoaSet.from_polish_model(engine, model, pm, PolishParams.shipped(), wl.drafts, wl.reads, wl.strands,
                                     wl.anchors, quals)
        s.set_device_steps(run_lengths=True, indels=device_indels)
        t0 = time.perf_counter()
        s.realign_all()
        s.estimate_repeat_counts()
        t1 = time.perf_counter()
        changed = sum(int(s.reference(c).chars != wl.drafts[c].chars) for c in range(s.n_chunks))
        phases = {k: round(v, 4) for k, v in s.phase_seconds().items()}
        s.close()
        if best is None or t1 - t0 < best["seconds"]:
            best = {"seconds": t1 - t0, "chunks_changed": changed, "phase_seconds": phases}
    best.update({"workload": "8 chunks x 10 kb (homopolymer-enriched), 50x, reads of 3-9 kb with base qualities, "
                             "drafts with 1% homopolymer-biased indels; no consensus iterations, one polish "
                             "iteration (params/allParams.np.json)",
                 "reads": int(sum(len(r) for r in wl.reads)),
                 "bases": int(sum(r.non_rle_length for lst in wl.reads for r in lst))})
    return best


def measure_polish(engine, model, pm):
    """The POA loop (poa_realignAll in consensus mode, up to 5 iterations) over 16 chunks of a
    homopolymer-enriched 10 kb template at 30x, reads of 3-9 kb, drafts with 1% indels."""
    from marginpolish_b200 import PoaSet, PolishParams, synth
    wl = synth.config_polish(seed=41, n_chunks=16, chunk_len=10_000, coverage=30, read_len=(3000, 9000),
                             hp_runs=True)
    pp = PolishParams(max_iterations=5)
    best = None
    for _ in range(2):
        s = PoaSet.from_polish_model(engine, model, pm, pp, wl.drafts, wl.reads, wl.strands, wl.anchors)
        t0 = time.perf_counter()
        s.realign()
        t1 = time.perf_counter()
        s.iterate()
        s.estimate_repeat_counts()
        t2 = time.perf_counter()
        its = [s.info(c)["iterations"] for c in range(s.n_chunks)]
        s.close()
        if best is None or t2 - t0 < best["seconds"]:
            best = {"seconds": t2 - t0, "realign_seconds": t1 - t0, "iterate_seconds": t2 - t1,
                    "iterations": its}
    best.update({"workload": "16 chunks x 10 kb (homopolymer-enriched), 30x, reads 3-9 kb, drafts with 1% "
                             "homopolymer-biased indels, up to 5 consensus iterations",
                 "reads": int(sum(len(r) for r in wl.reads)), "bases": int(sum(r.non_rle_length for lst in wl.reads
                                                                            for r in lst))})
    return best


def config_1mb():
    """The polishing loop at genome scale: 1 Mb as 10 chunks of 110 kb (100 kb plus 10 kb
    overlap; independent synthetic templates, since chunk stitching is outside this library),
    50x, log-normal reads (median 20 kb, sigma 0.6, at most 100 kb, clipped to the chunk), band
    half-width 64, drafts with 1% homopolymer-biased indels."""
    from marginpolish_b200 import synth
    return synth.config_polish(seed=47, n_chunks=10, chunk_len=110_000, coverage=50, half_width=64, hp_runs=True,
                               read_lognormal=(20_000, 0.6, 100_000))


def config_5mb(n_chunks=50):
    """The large-scale pass: 5 Mb as 50 independent chunks of 100 kb (homopolymer-enriched:
    geometric run lengths, p = 0.55), 60x, log-normal reads (median 25 kb, sigma 0.6, at most
    150 kb, clipped to the chunk), band half-width 96, drafts with 1% indels."""
    from marginpolish_b200 import synth
    return synth.config_polish(seed=53, n_chunks=n_chunks, chunk_len=100_000, coverage=60, half_width=96,
                               hp_runs=True, read_lognormal=(25_000, 0.6, 150_000))


def measure_realign_pass(engine, model, pm, wl, peak, cpu_seconds, plain_reads=16):
    """The first realignment pass of a polishing workload (every read against its chunk's draft)
    in the device-resident form of the headline: GCUPS (band + posterior kernels, CUDA events,
    inputs resident in HBM), the posterior kernel's FP32-roofline fraction, the plain
    one-read-per-launch form on its first reads, and the reference's own code (Oracle A) on all
    host cores on a bounded prefix of the same jobs (OpenMP over reads)."""
    import numpy as np
    from marginpolish_b200 import DeviceBatch
    t0 = time.perf_counter()
    jobs = wl.realign_workload().jobs()
    db = DeviceBatch(engine, model, pm.alignment, jobs)
    plan_s = time.perf_counter() - t0
    for _ in range(2):
        db.run()
    cells, n_tasks, _ = db.stats()
    ms, post = [], []
    for _ in range(5):
        ms.append(db.run())
        post.append(db.timing()[1])
    m, p = float(np.median(ms)), float(np.median(post))
    achieved = cells * FLOP_PER_CELL / (p * 1e-3) / 1e12
    p_ms, p_cells = db.run_plain(plain_reads)
    db.close()
    out = {"reads": jobs.n_jobs, "cells": cells, "tasks": n_tasks, "ms": m, "gcups": cells / (m * 1e-3) / 1e9,
           "posterior_ms": p,
           "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak},
           "plain_gpu": {"gcups": p_cells / (p_ms * 1e-3) / 1e9, "reads": min(plain_reads, n_tasks), "cells": p_cells},
           "plan_and_upload_s": round(plan_s, 2)}
    from oracle.bindings import RefOracle, available_reference
    if available_reference():
        ref = RefOracle()
        hf, hr = reference_models(ref, pm)
        cores = os.cpu_count() or 1
        pc = reference_cells(ref, job_prefix(jobs, min(jobs.n_jobs, 4 * cores)), pm)

        def run(n):
            t = time.perf_counter()
            ref.align_batch(hf, hr, job_prefix(jobs, n), pm.alignment, cores)
            return time.perf_counter() - t

        n = min(jobs.n_jobs, cores)
        t = run(n)
        rounds = max(1, min(4, int(round(cpu_seconds / max(t, 1e-3)))))
        n = min(jobs.n_jobs, cores * rounds)
        t = run(n)
        c = int(pc[:n].sum()) if n <= pc.size else int(reference_cells(ref, job_prefix(jobs, n), pm).sum())
        ref.free_model(hf)
        ref.free_model(hr)
        out["cpu_reference"] = {"gcups": c / t / 1e9, "cores": cores, "kind": "reference",
                                "sample": f"first {n} reads ({c} cells), OpenMP over reads on {cores} threads"}
        out["batched_over_reference"] = out["gcups"] / out["cpu_reference"]["gcups"]
    out["batched_over_plain"] = out["gcups"] / out["plain_gpu"]["gcups"]
    return out


def measure_polish_loop(engine, model, pm, wl, max_iterations, runs=2):
    """poa_realignAll in consensus mode over a polishing workload: the first realignment, then
    the consensus iterations, wall seconds with the per-phase split; the fastest of `runs` runs
    (the first run on an engine also grows its buffers), with the first run's time beside it."""
    from marginpolish_b200 import PoaSet, PolishParams
    best, first = None, None
    for _ in range(runs):
        s = PoaSet.from_polish_model(engine, model, pm, PolishParams(max_iterations=max_iterations), wl.drafts,
                                     wl.reads, wl.strands, wl.anchors)
        t0 = time.perf_counter()
        s.realign()
        t1 = time.perf_counter()
        s.iterate()
        s.estimate_repeat_counts()
        t2 = time.perf_counter()
        its = [s.info(c)["iterations"] for c in range(s.n_chunks)]
        phases = {k: round(v, 3) for k, v in s.phase_seconds().items()}
        s.close()
        r = {"seconds": t2 - t0, "realign_seconds": t1 - t0, "iterate_seconds": t2 - t1, "phase_seconds": phases,
             "iterations": its}
        first = r["seconds"] if first is None else first
        if best is None or r["seconds"] < best["seconds"]:
            best = r
    best.update({"first_run_seconds": first, "runs": runs, "chunks": len(wl.drafts),
                 "reads": int(sum(len(r) for r in wl.reads)),
                 "bases": int(sum(r.non_rle_length for lst in wl.reads for r in lst))})
    return best


def measure_scale_configs(engine, model, pm, peak, cpu_seconds, chunks_5mb):
    """The two larger configurations, reported beside the headline."""
    out = {}
    t = time.perf_counter()
    wl = config_1mb()
    gen = time.perf_counter() - t
    r = measure_realign_pass(engine, model, pm, wl, peak, cpu_seconds)
    r["workload"] = config_1mb.__doc__.split(".")[0].replace("\n", " ").replace("    ", " ")
    r["generation_s"] = round(gen, 1)
    r["polish_loop"] = measure_polish_loop(engine, model, pm, wl, 5)
    out["config_1mb_polish"] = r
    t = time.perf_counter()
    wl = config_5mb(chunks_5mb)
    gen = time.perf_counter() - t
    r = measure_realign_pass(engine, model, pm, wl, peak, cpu_seconds)
    r["workload"] = (config_5mb.__doc__.split(".")[0].replace("\n", " ").replace("    ", " ") +
                     (f" (the first {chunks_5mb} of its 50 chunks)" if chunks_5mb < 50 else ""))
    r["generation_s"] = round(gen, 1)
    out["config_5mb_pass"] = r
    return out


def pinned_jobs(jobs):
    """Copy of a batch whose arrays live in page-locked host memory (the library's allocator)."""
    from marginpolish_b200 import Jobs
    from marginpolish_b200.realign import pinned_empty

    arrs = {}
    for name in ("x_symbols", "x_begin", "x_end", "y_symbols", "y_offsets", "anchors", "anchor_offsets", "strand",
                 "x_shift"):
        v = getattr(jobs, name)
        if v is None:
            arrs[name] = None
            continue
        arr = pinned_empty(v.shape, v.dtype)
        arr[...] = v
        arrs[name] = arr
    return Jobs(arrs["x_symbols"], arrs["x_begin"], arrs["x_end"], arrs["y_symbols"], arrs["y_offsets"],
                arrs["anchors"], arrs["anchor_offsets"], arrs["strand"], None, None, arrs["x_shift"])


def run_ours(args, rank, world, local):
    import numpy as np
    import torch

    from marginpolish_b200 import DeviceBatch, Engine, Model, realign_batch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    pm = load_model()
    t0 = time.perf_counter()
    wl = make_workload(args, rank)
    jobs = wl.jobs()
    gen_s = time.perf_counter() - t0
    engine = Engine(local)
    engine.set_tuning(warps_per_block=args.warps, lanes_per_task=args.lanes)
    model = Model.from_polish(engine, pm)
    # autotuner: kernel variant (band tile, checkpoint stride) and warps per hull class, timed on
    # a separate sample of the same kind of batch (outside the timed region)
    tuned = None
    if args.autotune_chunks > 0 and args.lanes == 0 and args.warps == 0 and args.config == "batched":
        from marginpolish_b200 import synth
        t1 = time.perf_counter()
        sample = synth.config_batched(seed=args.seed + 1000 + rank, n_chunks=args.autotune_chunks).jobs()
        rep = engine.autotune(model, pm.alignment, sample)
        tuned = {"sample_chunks": args.autotune_chunks, "seconds": round(time.perf_counter() - t1, 1),
                 "classes": [{k: (round(r[k], 1) if k.endswith("gcups") else r[k])
                              for k in ("max_hull", "tasks", "candidates", "variant", "lanes_per_task",
                                        "cells_per_lane", "checkpoint_stride", "warps_per_block", "gcups",
                                        "default_gcups")} for r in rep if r["candidates"] > 0]}
    if not args.no_graphs:
        engine.set_graph_capture(True)
    db = DeviceBatch(engine, model, pm.alignment, jobs)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    for _ in range(args.warmup):
        db.run()
    cells, n_tasks, launches = db.stats()
    sampler = ClockSampler(local) if rank == 0 else None
    barrier()
    if sampler:
        sampler.start()
        time.sleep(0.4)
    dev_ms, post_ms, band_ms = [], [], []
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        ms = db.run()
        b, p = db.timing()
        dev_ms.append(ms)
        post_ms.append(p)
        band_ms.append(b)
    barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop() if sampler else None
    total_ms = float(sum(dev_ms))
    if dist is not None:
        t = torch.tensor([total_ms, float(cells)], dtype=torch.float64, device=f"cuda:{local}")
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = t.clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        max_ms, all_cells = float(mx[0]), float(sm[1])
    else:
        max_ms, all_cells = total_ms, float(cells)
    value = all_cells * args.steps / (max_ms * 1e-3) / 1e9
    # the timed run's results, for the FP64 check in the CPU-baseline leg (fetched before the
    # plain form reuses the batch)
    timed_res = db.fetch() if (rank == 0 and world == 1 and not args.no_cpu) else None

    # end-to-end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        from marginpolish_b200 import realign_batch_pipelined
        from marginpolish_b200.realign import OutputBuffer
        pj = pinned_jobs(jobs)
        out = OutputBuffer(pinned=True)  # page-locked result arrays, sized by the warm-up call
        realign_batch_pipelined(engine, model, pm.alignment, pj, out=out)  # warm (sizes the buffer)
        e2e_times = []
        h2d = int(pj.x_symbols.nbytes + pj.y_symbols.nbytes + pj.anchors.nbytes + pj.x_begin.nbytes * 2 +
                  pj.y_offsets.nbytes + pj.anchor_offsets.nbytes + pj.strand.nbytes + pj.x_shift.nbytes)
        d2h = 0
        steps_e2e = args.steps
        for _ in range(steps_e2e):
            barrier()
            t = time.perf_counter()
            r = realign_batch_pipelined(engine, model, pm.alignment, pj, out=out)
            torch.cuda.synchronize(local)
            e2e_times.append(time.perf_counter() - t)
            # tuples (weight, x, y), per-job offsets / likelihoods / cells, per-task statuses
            d2h = int(sum(int(r.offsets[k][-1]) for k in range(3)) * 12 + jobs.n_jobs * (3 * 8 + 16) + n_tasks * 32)
        e2e_t = max(e2e_times) if dist is None else e2e_times
        tt = float(np.median(e2e_times))
        if dist is not None:
            t = torch.tensor([tt], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tt = float(t[0])
        e2e = {"value": all_cells / tt / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": tt * 1e3,
               "form": "mp_realign_batch_into: host batch in, tuples out to page-locked arrays; job slices "
                       "alternate between two streams so copies overlap kernels"}
        del e2e_t

    # the plain one-read-per-launch form of the same kernel on the first reads of the batch
    plain = None
    if not args.no_plain and rank == 0:
        p_ms, p_cells = db.run_plain(args.plain_reads)
        plain = {"value": p_cells / (p_ms * 1e-3) / 1e9, "unit": "GCUPS", "reads": min(args.plain_reads, n_tasks),
                 "cells": p_cells, "ms": p_ms, "form": "one launch of one warp per read, same kernel and accuracy",
                 "batched_over_plain": (value / world) / (p_cells / (p_ms * 1e-3) / 1e9)}
    extras = {}
    if not args.no_extras and rank == 0:
        extras["adjoint"] = measure_adjoint(engine, model, pm)
        extras["polish_loop"] = measure_polish(engine, model, pm)
        extras["bubble_scoring"] = measure_bubble_scoring(engine, model, pm, cpu_sample=not args.no_cpu)
        extras["polish_loop_shipped"] = measure_polish_shipped(engine, model, pm)
    peak = engine.fp32_peak_tflops()
    if not args.no_scale and rank == 0 and world == 1 and args.config == "batched":
        # the larger configurations need the device memory the headline's buffers hold
        engine.release_buffers()
        try:
            extras.update(measure_scale_configs(engine, model, pm, peak, args.cpu_seconds / 2, args.chunks_5mb))
        except Exception as exc:  # reported in the line; the headline stands on its own
            extras["scale_configs_error"] = f"{type(exc).__name__}: {exc}"
    post = float(np.median(post_ms))
    achieved = cells * FLOP_PER_CELL / (post * 1e-3) / 1e12
    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu and world == 1:
            from oracle.bindings import available_reference
            if available_reference() and args.config == "batched":
                r = time_reference(pm, wl, jobs, args.cpu_seconds)
                cpu = {"value": r["gcups"], "unit": "GCUPS", "cores": r["cores"], "kind": "reference",
                       "sample": f"rate on a prefix of {r['chunks']} whole chunks ({r['reads']} reads, "
                                 f"{r['cells']} cells), OpenMP over chunks (schedule(dynamic,1)) on "
                                 f"{r['cores']} threads",
                       "value_1core": r["gcups_1core"],
                       "sample_1core": f"first chunk ({r['reads_1core']} reads), 1 thread",
                       "accuracy_of_timed_results": accuracy_sample(jobs, timed_res, pm)}
        line = {
            "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, shipped run-length model)",
            "config": {"workload": f"{args.config}: {wl.meta}", "reads": jobs.n_jobs, "cells_per_gpu_step": cells,
                       "tasks": n_tasks, "l2": "inputs and band/scratch/output buffers exceed the 126 MB L2",
                       "generation_s": round(gen_s, 1), "band_ms": float(np.median(band_ms)),
                       "posterior_ms": post, "wall_s_timed": wall,
                       "tuning": {"lanes_per_task": args.lanes or "auto", "warps_per_block": args.warps or "auto",
                                  "autotune": tuned},
                       "launch": "direct" if args.no_graphs else "CUDA graph replay of the pass's launches"},
            "e2e": e2e,
            "gpu_launches": launches * args.steps,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": DRAM_BYTES_PER_CELL * cells,
                         "traffic_note": "DRAM bytes per posterior launch: ncu bytes per cell x cells",
                         "note": f"{FLOP_PER_CELL} flop per cell x cells / posterior-kernel event time; "
                                 "peak = FP32 FMA throughput measured live on this GPU (mp_measure_fp32_peak)"},
            "cpu_baseline": cpu,
            "plain_gpu": plain,
            "clocks": clocks,
            **extras,
        }
        print(json.dumps(line), flush=True)
    db.close()
    model.close()
    engine.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
    elif args.polish_shipped:
        from marginpolish_b200 import Engine, Model, params
        pm = params.polish_model_from_npz(os.path.join(ROOT, "tests", "golden", "model_np.npz"))
        engine = Engine(local)
        model = Model.from_polish(engine, pm)
        print(json.dumps({"polish_loop_shipped": measure_polish_shipped(engine, model, pm, not args.host_indels)}),
              flush=True)
    elif args.bubble_scores:
        from marginpolish_b200 import Engine, Model, params
        pm = params.polish_model_from_npz(os.path.join(ROOT, "tests", "golden", "model_np.npz"))
        engine = Engine(local)
        model = Model.from_polish(engine, pm)
        print(json.dumps({"bubble_scoring": measure_bubble_scoring(engine, model, pm, cpu_sample=False)}), flush=True)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
