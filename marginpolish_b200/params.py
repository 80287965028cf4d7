"""Model and banding parameters of the realignment pass, loaded from MarginPolish
params JSON files (the reference's params/*.json format).

Lowering follows the reference's construction of the per-strand state machines:

* ``hmm_getStateMachine`` (impl/stateMachine.c:676-689): emissions are the logs
  of the 16 match / 4 gap-x / 4 gap-y probabilities (``emissions_construct``,
  :478-488); transitions are tied pairwise for the symmetric type
  (``stateMachine3_loadSymmetric``, :649-668) or taken as is for the asymmetric
  type (``stateMachine3_loadAsymmetric``, :632-647).
* reverse-strand reads use reverse-complemented emissions
  (``nucleotideEmissions_reverseComplement``, :454-470, applied by
  impl/parser.c:241-243): match[x][y] <- match[3-x][3-y], gap[x] <- gap[3-x].
* with ``useRepeatCountsInAlignment`` the match emission gains
  2.3025 * log10 R[base'][underlying][observed] (impl/stateMachine.c:718-722,
  swap at impl/parser.c:391-401; strand flag 1 for the forward machine, 0 for
  the reverse one); the table is parsed from ``repeatCountLogProbabilities_*_F``
  (impl/parser.c:99-152, layout [underlying][observed]).
* boundary vectors: start = match state only, ragged start = gap states only,
  end = transitions into match, ragged end = (gap-open average, gap extends)
  (impl/stateMachine.c:518-557).
* symbols with base >= 4 ('N') emit log(0.25^2) in a match and log(0.25) in a
  gap (impl/stateMachine.c:360-380); both constants are the reference's literals.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib

LOG_ZERO = -math.inf
# Literal log constants of the reference's ambiguous-base emissions (impl/stateMachine.c:362, :377).
N_GAP_LOG = -1.386294361
N_MATCH_LOG = -2.772588722
# Multiplier applied to the log10 repeat table (impl/stateMachine.c:721).
REPEAT_SCALE = 2.3025
MAX_REPEAT = 51  # inc/margin.h:123

MATCH, GAP_X, GAP_Y = 0, 1, 2
SYMMETRIC, ASYMMETRIC = 2, 3


def _log(p: float) -> float:
    return math.log(p) if p > 0 else LOG_ZERO


@dataclass
class StateModel:
    """A lowered 3-state machine for one read strand (all values natural logs)."""

    log_transitions: np.ndarray  # (9,) from*3+to
    log_start: np.ndarray
    log_ragged_start: np.ndarray
    log_end: np.ndarray
    log_ragged_end: np.ndarray
    log_match: np.ndarray  # (25,) [xbase*5 + ybase]
    log_gap_x: np.ndarray  # (5,)
    log_gap_y: np.ndarray  # (5,)
    run_length: bool = False
    strand: int = 1
    repeat_log10: Optional[np.ndarray] = None  # (4, 51, 51) [base][underlying][observed]
    repeat_scale: float = REPEAT_SCALE

    def desc(self) -> _lib.ModelDesc:
        """C struct for mp_model_create (keeps a reference to the repeat table)."""
        d = _lib.ModelDesc()
        d.log_transitions[:] = [float(v) for v in self.log_transitions]
        d.log_start[:] = [float(v) for v in self.log_start]
        d.log_ragged_start[:] = [float(v) for v in self.log_ragged_start]
        d.log_end[:] = [float(v) for v in self.log_end]
        d.log_ragged_end[:] = [float(v) for v in self.log_ragged_end]
        d.log_match[:] = [float(v) for v in self.log_match]
        d.log_gap_x[:] = [float(v) for v in self.log_gap_x]
        d.log_gap_y[:] = [float(v) for v in self.log_gap_y]
        d.run_length = 1 if self.run_length else 0
        d.strand = int(self.strand)
        d.max_repeat = MAX_REPEAT
        d.repeat_scale = float(self.repeat_scale)
        if self.run_length:
            tab = np.ascontiguousarray(self.repeat_log10, dtype=np.float64).reshape(-1)
            self._keep = tab
            d.repeat_log10 = _lib.ptr(tab, _lib.c_double)
        else:
            d.repeat_log10 = None
        return d


def machine_transitions(hmm_type: int, t: np.ndarray) -> np.ndarray:
    """Log transitions (from*3+to) of stateMachine3 loaded from a 3x3 probability matrix."""
    t = np.asarray(t, dtype=np.float64).reshape(3, 3)
    out = np.empty(9)
    if hmm_type == SYMMETRIC:
        mm = _log(t[MATCH, MATCH])
        to_m = _log((t[GAP_X, MATCH] + t[GAP_Y, MATCH]) / 2.0)
        opn = _log((t[MATCH, GAP_X] + t[MATCH, GAP_Y]) / 2.0)
        ext = _log((t[GAP_X, GAP_X] + t[GAP_Y, GAP_Y]) / 2.0)
        sw = _log((t[GAP_Y, GAP_X] + t[GAP_X, GAP_Y]) / 2.0)
        vals = {(MATCH, MATCH): mm, (GAP_X, MATCH): to_m, (GAP_Y, MATCH): to_m, (MATCH, GAP_X): opn,
                (MATCH, GAP_Y): opn, (GAP_X, GAP_X): ext, (GAP_Y, GAP_Y): ext, (GAP_Y, GAP_X): sw,
                (GAP_X, GAP_Y): sw}
    elif hmm_type == ASYMMETRIC:
        vals = {(a, b): _log(t[a, b]) for a in range(3) for b in range(3)}
    else:
        raise ValueError(f"unrecognised state machine type {hmm_type}")
    for (a, b), v in vals.items():
        out[a * 3 + b] = v
    return out


def boundary_vectors(lt: np.ndarray):
    """start, ragged start, end, ragged end (impl/stateMachine.c:518-557)."""
    start = np.array([0.0, LOG_ZERO, LOG_ZERO])
    ragged_start = np.array([LOG_ZERO, 0.0, 0.0])
    end = np.array([lt[MATCH * 3 + MATCH], lt[GAP_X * 3 + MATCH], lt[GAP_Y * 3 + MATCH]])
    ragged_end = np.array([(lt[MATCH * 3 + GAP_X] + lt[MATCH * 3 + GAP_Y]) / 2.0, lt[GAP_X * 3 + GAP_X],
                           lt[GAP_Y * 3 + GAP_Y]])
    return start, ragged_start, end, ragged_end


def build_state_model(hmm_type: int, transitions, emissions, reverse_complement: bool,
                      repeat_log10: Optional[np.ndarray] = None, strand: int = 1) -> StateModel:
    """Lowers an HMM (3x3 transition and 24 emission probabilities) to a StateModel."""
    lt = machine_transitions(hmm_type, transitions)
    em = np.asarray(emissions, dtype=np.float64)
    match = np.array([_log(v) for v in em[0:16]]).reshape(4, 4)
    gx = np.array([_log(v) for v in em[16:20]])
    gy = np.array([_log(v) for v in em[20:24]])
    if reverse_complement:
        match = match[::-1, ::-1].copy()
        gx = gx[::-1].copy()
        gy = gy[::-1].copy()
    m5 = np.full((5, 5), N_MATCH_LOG)
    m5[:4, :4] = match
    gx5 = np.append(gx, N_GAP_LOG)
    gy5 = np.append(gy, N_GAP_LOG)
    start, ragged_start, end, ragged_end = boundary_vectors(lt)
    return StateModel(lt, start, ragged_start, end, ragged_end, m5.reshape(-1), gx5, gy5,
                      run_length=repeat_log10 is not None, strand=strand,
                      repeat_log10=None if repeat_log10 is None else np.asarray(repeat_log10, dtype=np.float64))


@dataclass
class AlignmentParams:
    """PairwiseAlignmentParameters (inc/pairwiseAligner.h:28-39); defaults of
    pairwiseAlignmentBandingParameters_construct (impl/pairwiseAligner.c:999-1011)."""

    threshold: float = 0.01
    min_diags_between_traceback: int = 1000
    traceback_diagonals: int = 40
    diagonal_expansion: int = 20
    constraint_diagonal_trim: int = 14
    split_matrix_bigger_than_this: int = 3000 * 3000
    align_ambiguity_characters: bool = False
    gap_gamma: float = 0.5
    dynamic_anchor_expansion: bool = False

    def struct(self) -> _lib.Params:
        p = _lib.Params()
        p.threshold = self.threshold
        p.min_diags_between_traceback = self.min_diags_between_traceback
        p.traceback_diagonals = self.traceback_diagonals
        p.diagonal_expansion = self.diagonal_expansion
        p.constraint_diagonal_trim = self.constraint_diagonal_trim
        p.split_matrix_bigger_than_this = self.split_matrix_bigger_than_this
        p.dynamic_anchor_expansion = 1 if self.dynamic_anchor_expansion else 0
        p.gap_gamma = self.gap_gamma
        return p


_PARAM_KEYS = {
    "threshold": ("threshold", float),
    "minDiagsBetweenTraceBack": ("min_diags_between_traceback", int),
    "traceBackDiagonals": ("traceback_diagonals", int),
    "diagonalExpansion": ("diagonal_expansion", int),
    "constraintDiagonalTrim": ("constraint_diagonal_trim", int),
    "splitMatrixBiggerThanThis": ("split_matrix_bigger_than_this", int),
    "alignAmbiguityCharacters": ("align_ambiguity_characters", bool),
    "gapGamma": ("gap_gamma", float),
    "dynamicAnchorExpansion": ("dynamic_anchor_expansion", bool),
}


def parse_alignment_params(obj: dict) -> AlignmentParams:
    """pairwiseAlignmentParameters_jsonParse (impl/pairwiseAligner.c:1017-1066): unknown keys are an error."""
    p = AlignmentParams()
    for k, v in obj.items():
        if k not in _PARAM_KEYS:
            raise ValueError(f"Unrecognised key in pairwise alignment parameters json: {k}")
        name, typ = _PARAM_KEYS[k]
        setattr(p, name, typ(v))
    if p.diagonal_expansion % 2 != 0:
        raise ValueError("diagonalExpansion must be even")  # impl/parser.c:374
    return p


def parse_repeat_matrix(obj: dict) -> np.ndarray:
    """repeatSubMatrix_jsonParse (impl/parser.c:105-152): forward-strand tables per base."""
    tab = np.zeros((4, MAX_REPEAT, MAX_REPEAT))
    seen = set()
    for k, v in obj.items():
        if k in ("baseLogRepeatCounts_AT", "baseLogRepeatCounts_GC"):
            continue
        if len(k) != 31:
            raise ValueError(f"Unrecognised key in repeat sub matrix json: {k}")
        base, strand = k[28], k[30]
        if base not in "ACGT":
            raise ValueError(f"Unrecognised base in repeat sub matrix json: {k}")
        if strand != "F":
            raise ValueError(f"Unrecognised strand in repeat sub matrix json: {k}")
        arr = np.asarray(v, dtype=np.float64)
        if arr.size != MAX_REPEAT * MAX_REPEAT:
            raise ValueError(f"repeat matrix {k} has {arr.size} entries, expected {MAX_REPEAT ** 2}")
        tab["ACGT".index(base)] = arr.reshape(MAX_REPEAT, MAX_REPEAT)
        seen.add(base)
    return tab


@dataclass
class PolishModel:
    """The read-to-reference machines of a MarginPolish params file."""

    forward: StateModel
    reverse: StateModel
    alignment: AlignmentParams
    use_run_length_encoding: bool = True
    use_repeat_counts: bool = True
    repeat_log10: Optional[np.ndarray] = None
    raw: dict = field(default_factory=dict, repr=False)


def load_polish_model(path: str) -> PolishModel:
    """Reads a MarginPolish params JSON (the ``polish`` section) into a PolishModel."""
    with open(path) as fh:
        js = json.load(fh)
    pol = js["polish"] if "polish" in js else js
    hmm = pol["hmmForwardStrandReadGivenReference"]
    use_rle = bool(pol.get("useRunLengthEncoding", False))
    use_rc = bool(pol.get("useRepeatCountsInAlignment", False))
    if use_rc and not use_rle:
        raise ValueError("Trying to use repeat counts in read to reference alignment but not using run length encoding")
    rep = parse_repeat_matrix(pol["repeatCountSubstitutionMatrix"]) if "repeatCountSubstitutionMatrix" in pol else None
    if use_rc and rep is None:
        raise ValueError("repeat counts requested but no repeatCountSubstitutionMatrix given")
    ap = parse_alignment_params(pol["pairwiseAlignmentParameters"])
    fwd = build_state_model(int(hmm["type"]), hmm["transitions"], hmm["emissions"], False,
                            rep if use_rc else None, strand=1)
    rev = build_state_model(int(hmm["type"]), hmm["transitions"], hmm["emissions"], True,
                            rep if use_rc else None, strand=0)
    return PolishModel(fwd, rev, ap, use_rle, use_rc, rep, raw=pol)


def polish_model_from_tables(hmm_type: int, transitions, emissions, repeat_log10, alignment: AlignmentParams,
                             use_repeat_counts: bool = True) -> PolishModel:
    """PolishModel from raw tables (the HMM probabilities and the log10 repeat table)."""
    rep = np.asarray(repeat_log10, dtype=np.float64) if use_repeat_counts else None
    fwd = build_state_model(int(hmm_type), transitions, emissions, False, rep, strand=1)
    rev = build_state_model(int(hmm_type), transitions, emissions, True, rep, strand=0)
    return PolishModel(fwd, rev, alignment, True, use_repeat_counts, rep)


def polish_model_from_npz(path: str) -> PolishModel:
    """Reads a model fixture written by tests/golden/make_golden.py."""
    z = np.load(path)
    ap = AlignmentParams(threshold=float(z["threshold"]), min_diags_between_traceback=int(z["min_diags"]),
                         traceback_diagonals=int(z["traceback_diags"]), diagonal_expansion=int(z["diagonal_expansion"]),
                         constraint_diagonal_trim=int(z["constraint_trim"]),
                         split_matrix_bigger_than_this=int(z["split"]), dynamic_anchor_expansion=bool(z["dynamic"]),
                         gap_gamma=float(z["gap_gamma"]))
    return polish_model_from_tables(int(z["hmm_type"]), z["transitions"], z["emissions"], z["repeat_log10"], ap,
                                    bool(z["use_repeat_counts"]))


def default_state_model(transitions, match, gap, boundary) -> StateModel:
    """StateModel from tables of the reference's code-default machine (impl/stateMachine.c:598-630),
    as probed from the reference build: 9 log transitions, 25 log match emissions, 5x2 log gap emissions,
    4x3 boundary vectors (start, ragged start, end, ragged end)."""
    gap = np.asarray(gap, dtype=np.float64).reshape(5, 2)
    b = np.asarray(boundary, dtype=np.float64).reshape(4, 3)
    return StateModel(np.asarray(transitions, dtype=np.float64), b[0], b[1], b[2], b[3],
                      np.asarray(match, dtype=np.float64), gap[:, 0].copy(), gap[:, 1].copy(), run_length=False)


# The reference's code-default 3-state nucleotide machine, which removeOverlap aligns chunk
# overlaps with (stateMachine3_constructNucleotide, impl/polisher.c:1958-1959): the transition
# constants of impl/stateMachine.c:598-608 and the nucleotide emission tables of
# nucleotideEmissions_construct, as natural logs (tests/test_model.py pins them against the
# reference build). Transitions are from*3+to over (match, gap-x, gap-y); emissions by base
# A C G T N.
CODE_DEFAULT_TRANSITIONS = (
    -0.030064059121770816, -4.21256642, -4.21256642,
    -1.272871422049609, -0.3388262689231553, -4.910694825551255,
    -1.272871422049609, -4.910694825551255, -0.3388262689231553)
CODE_DEFAULT_MATCH = (
    -1.8917761142, -4.3459578861, -3.760242452, -4.3459578861, -2.772588722,
    -4.3459578861, -1.8917761142, -4.3459578861, -3.760242452, -2.772588722,
    -3.760242452, -4.3459578861, -1.8917761142, -4.3459578861, -2.772588722,
    -4.3459578861, -3.760242452, -4.3459578861, -1.8917761142, -2.772588722,
    -2.772588722, -2.772588722, -2.772588722, -2.772588722, -2.772588722)
CODE_DEFAULT_GAP = (  # (gap-x, gap-y) per base
    (-1.3862943611, -1.3862943611), (-1.3862943611, -1.3862943611), (-1.3862943611, -1.3862943611),
    (-1.3862943611, -1.3862943611), (-1.386294361, -1.386294361))
CODE_DEFAULT_BOUNDARY = (  # start, ragged start, end, ragged end
    (0.0, -np.inf, -np.inf), (-np.inf, 0.0, 0.0),
    (-0.030064059121770816, -1.272871422049609, -1.272871422049609),
    (-4.21256642, -0.3388262689231553, -0.3388262689231553))


def code_default_state_model() -> StateModel:
    """The code-default nucleotide machine (see CODE_DEFAULT_TRANSITIONS)."""
    return default_state_model(CODE_DEFAULT_TRANSITIONS, CODE_DEFAULT_MATCH, CODE_DEFAULT_GAP, CODE_DEFAULT_BOUNDARY)