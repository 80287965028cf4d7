"""Lowering of the reference's state machines to flat tables, against the reference's own machine
(Oracle A) evaluated on every symbol pair."""
import ctypes
import os

import numpy as np
import pytest

from marginpolish_b200 import params
from oracle.bindings import MpoModel

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "model_np.npz")


def _symbols():
    for b in range(5):
        for rc in (0, 1, 2, 7, 50):
            yield (rc << 8) | b


def test_lowered_run_length_model_matches_reference_machine(ref_oracle, exact_oracle, polish_model):
    z = np.load(GOLDEN)
    for rev, sm in ((False, polish_model.forward), (True, polish_model.reverse)):
        h = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], rev, z["repeat_log10"],
                             0 if rev else 1)
        assert np.array_equal(ref_oracle.transitions(h), sm.log_transitions)
        for which, vec in enumerate((sm.log_start, sm.log_ragged_start, sm.log_end, sm.log_ragged_end)):
            assert np.array_equal(ref_oracle.boundary(h, which), vec)
        m = MpoModel.from_state_model(sm)
        for cx in _symbols():
            gx, gy = ref_oracle.gap_emissions(h, cx)
            assert gx == exact_oracle.lib.mpo_gap_x_emission(ctypes.byref(m), cx)
            assert gy == exact_oracle.lib.mpo_gap_y_emission(ctypes.byref(m), cx)
            for cy in _symbols():
                assert ref_oracle.match_emission(h, cx, cy) == exact_oracle.lib.mpo_match_emission(ctypes.byref(m), cx, cy)
        ref_oracle.free_model(h)


def test_asymmetric_and_default_machines(ref_oracle):
    rng = np.random.default_rng(3)
    t = rng.random((3, 3))
    t /= t.sum(axis=1, keepdims=True)
    e = rng.random(24)
    for hmm_type in (params.SYMMETRIC, params.ASYMMETRIC):
        sm = params.build_state_model(hmm_type, t.reshape(-1), e, False, None)
        h = ref_oracle.model(hmm_type, t.reshape(-1), e, False, None, 1)
        assert np.array_equal(ref_oracle.transitions(h), sm.log_transitions)
        ref_oracle.free_model(h)
    z = np.load(GOLDEN)
    d = ref_oracle.default_model()
    assert np.array_equal(ref_oracle.transitions(d), z["default_transitions"])
    ref_oracle.free_model(d)


def test_code_default_machine_is_the_reference_build(ref_oracle, exact_oracle):
    """The library's code-default nucleotide machine (params.code_default_state_model, which
    chunk stitching uses) against the reference build's stateMachine3_constructNucleotide,
    table by table and on every symbol pair."""
    sm = params.code_default_state_model()
    d = ref_oracle.default_model()
    assert np.array_equal(ref_oracle.transitions(d), sm.log_transitions)
    for which, vec in enumerate((sm.log_start, sm.log_ragged_start, sm.log_end, sm.log_ragged_end)):
        assert np.array_equal(ref_oracle.boundary(d, which), vec)
    m = MpoModel.from_state_model(sm)
    for cx in range(5):
        gx, gy = ref_oracle.gap_emissions(d, cx)
        assert gx == exact_oracle.lib.mpo_gap_x_emission(ctypes.byref(m), cx)
        assert gy == exact_oracle.lib.mpo_gap_y_emission(ctypes.byref(m), cx)
        for cy in range(5):
            assert ref_oracle.match_emission(d, cx, cy) == exact_oracle.lib.mpo_match_emission(ctypes.byref(m), cx, cy)
    ref_oracle.free_model(d)


def test_params_json_parsing_rejects_unknown_keys():
    with pytest.raises(ValueError):
        params.parse_alignment_params({"threshold": 0.1, "bogus": 1})
    with pytest.raises(ValueError):
        params.parse_alignment_params({"diagonalExpansion": 3})
    p = params.parse_alignment_params({"threshold": 0.2, "dynamicAnchorExpansion": True})
    assert p.threshold == 0.2 and p.dynamic_anchor_expansion


def test_drop_in_lowering_through_the_state_machine_vtable(ref_oracle, polish_model):
    """mpd_lower_state_machine reads the caller's StateMachine through its function pointers only."""
    from marginpolish_b200 import _lib
    from oracle.bindings import SHIM_LIB
    ctypes.CDLL(SHIM_LIB, mode=ctypes.RTLD_GLOBAL)  # stands in for the host application's sonLib
    lib = ctypes.CDLL(os.path.join(os.path.dirname(_lib.LIB_PATH), "libmpgpu_dropin.so"))
    lib.mpd_lower_state_machine.restype = ctypes.c_int
    lib.mpd_lower_state_machine.argtypes = [ctypes.c_void_p, ctypes.POINTER(_lib.ModelDesc), ctypes.POINTER(ctypes.c_double)]
    z = np.load(GOLDEN)
    for rev, sm in ((False, polish_model.forward), (True, polish_model.reverse)):
        h = ref_oracle.model(int(z["hmm_type"]), z["transitions"], z["emissions"], rev, z["repeat_log10"],
                             0 if rev else 1)
        machine = ctypes.cast(h, ctypes.POINTER(ctypes.c_void_p))[0]  # RefoModel.sM (first field)
        d = _lib.ModelDesc()
        rep = np.zeros(4 * 51 * 51)
        assert lib.mpd_lower_state_machine(machine, ctypes.byref(d), _lib.ptr(rep, ctypes.c_double)) == 0
        assert d.run_length == 1
        assert np.array_equal(np.array(d.log_transitions[:]), sm.log_transitions)
        # reconstruct every match emission and compare with the reference's
        for cx in _symbols():
            for cy in _symbols():
                xb, rx, yb, ry = min(cx & 255, 4), cx >> 8, min(cy & 255, 4), cy >> 8
                row = 0 if xb == 4 else xb
                got = d.log_match[xb * 5 + yb] + rep[(row * 51 + rx) * 51 + ry]
                want = ref_oracle.match_emission(h, cx, cy)
                assert abs(got - want) <= 1e-9 * (1 + abs(want))
        ref_oracle.free_model(h)
