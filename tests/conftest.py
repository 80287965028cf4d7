"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on the CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")

# The drop-in library raises CUDA's hardware work queues to 32 when a host application loads it
# before creating its CUDA context; this test process creates its context first, so it asks
# for the same here, before any CUDA call.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def polish_model():
    from marginpolish_b200 import params
    return params.polish_model_from_npz(os.path.join(GOLDEN, "model_np.npz"))


@pytest.fixture(scope="session")
def default_model():
    """The reference's code-default nucleotide machine (tables probed from the reference build)."""
    from marginpolish_b200 import params
    z = np.load(os.path.join(GOLDEN, "model_np.npz"))
    return params.default_state_model(z["default_transitions"], z["default_match"], z["default_gap"],
                                      z["default_boundary"])


@pytest.fixture(scope="session")
def exact_oracle():
    from oracle.bindings import ExactOracle
    return ExactOracle()


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle.bindings import RefOracle, available_reference
    if not available_reference():
        pytest.skip("reference build (oracle/_ref) not present")
    return RefOracle()


@pytest.fixture(scope="session")
def engine():
    from marginpolish_b200 import Engine
    return Engine(0)
