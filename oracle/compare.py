"""Parity checks of the CUDA library against the oracles -- TEST INFRASTRUCTURE ONLY.

``check_job`` compares one job's GPU tuples with Oracle B's FP64 dense
posteriors (every band cell of every posterior diagonal):

* every emitted GPU tuple: |weight/1e7 - p_oracle| <= POSTERIOR_TOL (+1e-7 for
  the floor) and p_oracle >= threshold - POSTERIOR_TOL;
* every oracle posterior >= threshold + POSTERIOR_TOL is emitted by the GPU;
* the order of the tuples both emit is identical (the reference's order);
* the log-likelihood agrees within LOGLIK_TOL (relative to |log L|).
"""
from __future__ import annotations

import numpy as np

POSTERIOR_TOL = 1e-4
LOGLIK_REL_TOL = 1e-5


def dense_table(dense: np.ndarray):
    """(x, y) -> (pM, pX, pY) from Oracle B's dense records."""
    d = {}
    for r in dense:
        d[(int(r[0]), int(r[1]))] = (r[2], r[3], r[4])
    return d


def check_job(gpu_lists, oracle_out, threshold, tol=POSTERIOR_TOL):
    """Returns a report dict; raises AssertionError on a parity failure."""
    table = dense_table(oracle_out["dense"])
    max_err = 0.0
    n_gpu = 0
    for k in range(3):
        g = np.asarray(gpu_lists[k]).reshape(-1, 3)
        o = np.asarray(oracle_out["pairs"][k]).reshape(-1, 3)
        n_gpu += g.shape[0]
        gkeys = [(int(x), int(y)) for _, x, y in g]
        for (w, x, y) in g:
            rec = table.get((int(x), int(y)))
            assert rec is not None, f"list {k}: GPU tuple ({x}, {y}) is not a band cell of the oracle"
            p = rec[k]
            assert p >= 0.0, f"list {k}: GPU tuple ({x}, {y}) for an undefined state"
            err = abs(w / 1e7 - min(p, 1.0))
            max_err = max(max_err, err)
            assert err <= tol + 1e-7, f"list {k}: posterior at ({x}, {y}) GPU {w / 1e7} vs FP64 {p}"
            assert p >= threshold - tol, f"list {k}: GPU emitted ({x}, {y}) with FP64 posterior {p}"
        gset = set(gkeys)
        # every clearly-above-threshold oracle cell is emitted
        for key, rec in table.items():
            p = rec[k]
            if p >= threshold + tol:
                assert key in gset, f"list {k}: FP64 posterior {p} at {key} missing from GPU output"
        # common tuples appear in the same order
        okeys = [(int(x), int(y)) for _, x, y in o]
        oset = set(okeys)
        common_g = [kk for kk in gkeys if kk in oset]
        common_o = [kk for kk in okeys if kk in gset]
        assert common_g == common_o, f"list {k}: tuple order differs from the reference order"
    ll_ref = oracle_out["log_likelihood"]
    return {"max_abs_posterior_error": max_err, "tuples": n_gpu, "loglik_oracle": ll_ref}


def check_loglik(gpu_ll, oracle_ll, rel=LOGLIK_REL_TOL):
    err = abs(gpu_ll - oracle_ll)
    assert err <= rel * max(1.0, abs(oracle_ll)), f"log-likelihood GPU {gpu_ll} vs FP64 {oracle_ll}"
    return err


def set_diff_against_reference(gpu_lists, ref_lists, oracle_out, threshold, band=1e-4):
    """Pairs in one of GPU / reference (Oracle A) but not the other must lie within `band` of the threshold
    (the reference's approximate logAdd moves posteriors near 0.01 by < 1e-5). Returns the number of
    differing tuples."""
    table = dense_table(oracle_out["dense"])
    ndiff = 0
    for k in range(3):
        g = {(int(x), int(y)) for _, x, y in np.asarray(gpu_lists[k]).reshape(-1, 3)}
        r = {(int(x), int(y)) for _, x, y in np.asarray(ref_lists[k]).reshape(-1, 3)}
        for key in g ^ r:
            rec = table.get(key)
            assert rec is not None, f"list {k}: {key} differs from the reference, far below the threshold in FP64"
            p = rec[k]
            assert abs(p - threshold) <= band, f"list {k}: {key} differs from the reference with FP64 p={p}"
            ndiff += 1
    return ndiff
