import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding

    if not os.path.exists(binding.ORACLE_SO):
        binding.build(ref=False)
    return binding.Oracle()


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle import binding

    if not os.path.exists(binding.REF_SO):
        pytest.skip("oracle/_ref (the reference compiled from its sources) is not built here")
    return binding.RefOracle(binding.REF_SO)


@pytest.fixture(scope="session")
def golden_kernels():
    return dict(np.load(os.path.join(GOLDEN, "kernels.npz")))


@pytest.fixture(scope="session")
def golden_topology():
    return dict(np.load(os.path.join(GOLDEN, "topology.npz")))


def rel_err(got, ref) -> float:
    """max |got - ref| / max |ref|: the relative error measure of every parity test."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = float(np.max(np.abs(ref))) if ref.size else 0.0
    return float(np.max(np.abs(got - ref)) / max(scale, 1e-30)) if ref.size else 0.0


def bit_exact(got, ref) -> bool:
    return np.array_equal(np.asarray(got), np.asarray(ref))
