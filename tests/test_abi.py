"""The C ABI: every declared entry point is exported, and host-side paths behave without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from marginpolish_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header, prefix):
    """Function prototypes of a header whose names start with one of the given prefixes."""
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_]\w*)\s*\([^;{()]*(?:\([^()]*\)[^;{()]*)*\)\s*;", text)
    return sorted({n for n in names if n.startswith(prefix)})


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared("mpgpu.h", ("mp_",))
    assert "mp_realign_batch" in names and len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(_lib.EXPORTED) <= set(names)


def test_drop_in_exports_reference_signatures():
    dropin = os.path.join(os.path.dirname(_lib.LIB_PATH), "libmpgpu_dropin.so")
    out = os.popen(f"nm -D --defined-only {dropin}").read()
    names = _declared("mpgpu_dropin.h", ("get", "mpd_", "compute"))
    assert len(names) == 8 and "computeForwardProbability" in names and "getExpectationsUsingAnchors" in names
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n
    undefined = os.popen(f"nm -D --undefined-only {dropin}").read()
    assert "stList_append" in undefined  # resolved from the host application's sonLib


def test_engine_without_gpu_reports_cuda_error():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.mp_engine_create(0, ctypes.byref(h))
    assert st == _lib.MP_ERR_CUDA
    assert lib.mp_last_error()


def test_geometry_helpers_validate_arguments():
    lib = _lib.load()
    out = np.zeros((4, 3), dtype=np.int64)
    assert lib.mp_band(None, 0, -1, 2, 0, 0, _lib.ptr(out, ctypes.c_int64)) == _lib.MP_ERR_ARGUMENT
    s, e = ctypes.c_int64(), ctypes.c_int64()
    a = np.array([[5, 0, 0]], np.int32)
    # crop range beyond the template is an error
    assert lib.mp_crop_range(_lib.ptr(a, ctypes.c_int32), 1, 3, 10, s, e) == _lib.MP_ERR_ARGUMENT
