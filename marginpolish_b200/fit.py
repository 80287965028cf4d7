"""Validation and parameter-fitting harness around the adjoint kernel.

Not part of the realignment path: it wraps mp_expectations_batch (the gradient of the
summed read log-likelihood with respect to the log parameters, i.e. the Baum-Welch
expected counts) in a torch.autograd.Function so that the pair HMM's parameters can be
fitted by gradient descent, and so the gradient can be checked against finite differences.

Parameterisation (the reference's model, impl/stateMachine.c:360-380, :518-557, :632-668,
:702-736): a 3x3 transition matrix (rows normalised), 4x4 match emissions (normalised over
the 16 pairs), 4 gap-x and 4 gap-y emissions, and the [4][51][51] run-length table
(normalised over the observed count for each base and underlying count). Reverse-strand
reads use the reverse-complemented emissions (impl/stateMachine.c:454-470). The end
probabilities are functions of the transitions (end = the transitions into match); the
likelihood is over jobs without ragged ends.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from .params import N_GAP_LOG, N_MATCH_LOG, StateModel, boundary_vectors
from .realign import Engine, Jobs, Model, expectations_batch

REPEAT_SCALE = 2.3025


def _torch():
    import torch
    return torch


@dataclass
class FitParams:
    """Free parameters (unnormalised logits) of the pair HMM."""
    trans: "object"    # (3, 3) logits, row-normalised
    match: "object"    # (16,) logits over (x base, y base)
    gap_x: "object"    # (4,)
    gap_y: "object"    # (4,)
    repeat: "object"   # (4, 51, 51) logits, normalised over the observed count

    def tensors(self):
        return [self.trans, self.match, self.gap_x, self.gap_y, self.repeat]


def log_tables(p: FitParams):
    """Normalised natural-log tables of both strands' machines from the logits:
    (log transitions (2, 9), log match (2, 25), log gap-x (2, 5), log gap-y (2, 5), log run-length table
    (4, 51, 51) in natural-log units)."""
    torch = _torch()
    lt = torch.log_softmax(p.trans, dim=1).reshape(9)
    lm = torch.log_softmax(p.match, dim=0).reshape(4, 4)
    lgx = torch.log_softmax(p.gap_x, dim=0)
    lgy = torch.log_softmax(p.gap_y, dim=0)
    lrep = torch.log_softmax(p.repeat, dim=2)

    def five(m4):  # 'N' rows and columns keep the reference's constants
        out = torch.full((5, 5), N_MATCH_LOG, dtype=m4.dtype)
        out[:4, :4] = m4
        return out.reshape(25)

    def gap5(g):
        return torch.cat([g, torch.tensor([N_GAP_LOG], dtype=g.dtype)])

    match = torch.stack([five(lm), five(torch.flip(lm, [0, 1]))])
    gx = torch.stack([gap5(lgx), gap5(torch.flip(lgx, [0]))])
    gy = torch.stack([gap5(lgy), gap5(torch.flip(lgy, [0]))])
    return torch.stack([lt, lt]), match, gx, gy, lrep


def _state_model(lt, match, gx, gy, lrep, strand) -> StateModel:
    lt = np.asarray(lt, dtype=np.float64)
    start, ragged_start, end, ragged_end = boundary_vectors(lt)
    return StateModel(lt, start, ragged_start, end, ragged_end, np.asarray(match, np.float64),
                      np.asarray(gx, np.float64), np.asarray(gy, np.float64), run_length=True, strand=strand,
                      repeat_log10=np.asarray(lrep, np.float64) / REPEAT_SCALE, repeat_scale=REPEAT_SCALE)


class SummedLogLikelihood:
    """torch.autograd.Function over (log transitions, log match, log gap-x, log gap-y, log run-length
    table) of both strands: forward = sum of ln P over the jobs, backward = the expected counts."""

    @staticmethod
    def apply(lt, match, gx, gy, lrep, engine: Engine, jobs: Jobs, params):
        return _function().apply(lt, match, gx, gy, lrep, engine, jobs, params)


_FN = None


def _function():
    global _FN
    if _FN is not None:
        return _FN
    torch = _torch()

    class Fn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, lt, match, gx, gy, lrep, engine, jobs, params):
            if (jobs.ragged_left is not None and np.any(jobs.ragged_left)) or \
                    (jobs.ragged_right is not None and np.any(jobs.ragged_right)):
                raise ValueError("the harness fits jobs without ragged ends")
            t = [v.detach().cpu().double().numpy() for v in (lt, match, gx, gy, lrep)]
            fwd = _state_model(t[0][0], t[1][0], t[2][0], t[3][0], t[4], 1)
            rev = _state_model(t[0][1], t[1][1], t[2][1], t[3][1], t[4], 0)
            model = Model(engine, fwd, rev)
            try:
                ex = expectations_batch(engine, model, params, jobs)
            finally:
                model.close()
            g_lt = ex.transitions.reshape(2, 9).copy()
            # end = (t[M->M], t[X->M], t[Y->M]): its posterior adds to those transitions
            g_lt[:, 0] += ex.end[:, 0]
            g_lt[:, 3] += ex.end[:, 1]
            g_lt[:, 6] += ex.end[:, 2]
            grads = [torch.from_numpy(g_lt), torch.from_numpy(ex.match.reshape(2, 25).copy()),
                     torch.from_numpy(ex.gap_x.copy()), torch.from_numpy(ex.gap_y.copy()),
                     torch.from_numpy(ex.repeat[0].copy())]
            ctx.save_for_backward(*grads)
            return torch.tensor(ex.log_likelihood, dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            grads = [g * v for v in ctx.saved_tensors]
            return (*grads, None, None, None)

    _FN = Fn
    return Fn


def fit(engine: Engine, jobs: Jobs, params, init: FitParams, steps: int = 20, lr: float = 0.05,
        callback: Optional[callable] = None):
    """Adam on the negative mean log-likelihood per read; returns the per-step log-likelihoods."""
    torch = _torch()
    opt = torch.optim.Adam(init.tensors(), lr=lr)
    history = []
    for step in range(steps):
        opt.zero_grad()
        tables = log_tables(init)
        ll = SummedLogLikelihood.apply(*tables, engine, jobs, params)
        loss = -ll / max(jobs.n_jobs, 1)
        loss.backward()
        opt.step()
        value = float(ll.detach())
        history.append(value)
        if callback:
            callback(step, value)
    return history


def params_from_model(hmm_transitions, emissions, repeat_log10, perturb: float = 0.0, seed: int = 0) -> FitParams:
    """Logits reproducing a shipped model (3x3 transition probabilities, 24 emission
    probabilities, log10 run-length table), optionally perturbed by Gaussian noise."""
    torch = _torch()
    rng = np.random.default_rng(seed)

    def logit(p):
        a = np.log(np.maximum(np.asarray(p, np.float64), 1e-300))
        if perturb:
            a = a + perturb * rng.standard_normal(a.shape)
        return torch.tensor(a, dtype=torch.float64, requires_grad=True)

    t = np.asarray(hmm_transitions, np.float64).reshape(3, 3)
    em = np.asarray(emissions, np.float64)
    rep = 10.0 ** (REPEAT_SCALE / np.log(10.0) * np.asarray(repeat_log10, np.float64))
    return FitParams(logit(t), logit(em[:16]), logit(em[16:20]), logit(em[20:24]), logit(rep))
