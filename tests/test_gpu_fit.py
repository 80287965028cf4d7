"""The adjoint wrapped in torch.autograd (marginpolish_b200.fit): the gradient of the summed
log-likelihood with respect to the model's logits matches central finite differences of the
FP64 oracle's log-likelihood, and 20 Adam steps from perturbed parameters raise the
likelihood of the reads."""
import os

import numpy as np
import pytest

from marginpolish_b200 import synth
from marginpolish_b200.fit import _state_model, fit, log_tables, params_from_model, SummedLogLikelihood
from oracle.bindings import MpoModel

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def tables():
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    return z["transitions"], z["emissions"], z["repeat_log10"]


def _oracle_ll(exact_oracle, params, jobs, ap):
    lt, m, gx, gy, lrep = [v.detach().numpy() for v in log_tables(params)]
    total = 0.0
    for j in range(jobs.n_jobs):
        md = 0 if jobs.strand[j] else 1
        sm = _state_model(lt[md], m[md], gx[md], gy[md], lrep, 1 if md == 0 else 0)
        mpo = MpoModel.from_state_model(sm)
        sx = jobs.x_symbols[jobs.x_begin[j]:jobs.x_end[j]]
        sy = jobs.y_symbols[jobs.y_offsets[j]:jobs.y_offsets[j + 1]]
        a = jobs.anchors[jobs.anchor_offsets[j]:jobs.anchor_offsets[j + 1]]
        total += exact_oracle.forward_probability(mpo, sx, sy, a, ap.diagonal_expansion, True)
    return total


def test_autograd_gradient_matches_finite_differences(engine, polish_model, exact_oracle, tables):
    import torch
    ap = polish_model.alignment
    jobs = synth.config_small(seed=47, n_reads=2, template_len=500).jobs()
    p = params_from_model(*tables, perturb=0.05, seed=1)
    ll = SummedLogLikelihood.apply(*log_tables(p), engine, jobs, ap)
    ll.backward()
    assert float(ll.detach()) == pytest.approx(_oracle_ll(exact_oracle, p, jobs, ap), rel=1e-5)
    h = 1e-4
    probes = [(p.trans, (0, 1)), (p.trans, (1, 1)), (p.trans, (2, 0)), (p.match, (5,)), (p.match, (2,)),
              (p.gap_x, (1,)), (p.gap_y, (3,))]
    rep_grad = p.repeat.grad.numpy()
    probes += [(p.repeat, tuple(int(v) for v in np.unravel_index(np.argmax(np.abs(rep_grad)), rep_grad.shape)))]
    for t, idx in probes:
        with torch.no_grad():
            v0 = t[idx].item()
            t[idx] = v0 + h
            up = _oracle_ll(exact_oracle, p, jobs, ap)
            t[idx] = v0 - h
            dn = _oracle_ll(exact_oracle, p, jobs, ap)
            t[idx] = v0
        fd = (up - dn) / (2 * h)
        g = t.grad[idx].item()
        assert abs(g - fd) <= max(2e-3, 2e-3 * abs(fd)), (idx, g, fd)


def test_twenty_steps_of_fitting_raise_the_likelihood(engine, polish_model, tables):
    ap = polish_model.alignment
    jobs = synth.config_small(seed=53, n_reads=24, template_len=2500).jobs()
    p = params_from_model(*tables, perturb=0.3, seed=2)
    hist = fit(engine, jobs, ap, p, steps=20, lr=0.05)
    assert len(hist) == 20
    assert hist[-1] > hist[0] + 0.01 * abs(hist[0])
