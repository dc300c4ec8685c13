import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _have_gpu() -> bool:
    try:
        import universal_classical_montecarlo_b200 as u

        return u.device_count() > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device on this host")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import ORACLE_SO, Oracle, build

    if not os.path.isfile(ORACLE_SO):
        build(reference_root=None)
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Reference, have_reference

    if not have_reference():
        pytest.skip("reference harness (oracle/_ref) not built")
    return Reference()


@pytest.fixture(scope="session")
def umc():
    import universal_classical_montecarlo_b200 as u

    return u


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    path = os.path.join(GOLDEN, "golden.npz")
    if not os.path.isfile(path):
        pytest.skip("golden fixtures missing")
    return dict(np.load(path))
