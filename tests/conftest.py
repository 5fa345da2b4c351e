import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
TESTS = Path(__file__).resolve().parent
if str(TESTS) not in sys.path:
    sys.path.insert(0, str(TESTS))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running (full-size workloads)")


@pytest.fixture(scope="session")
def engine_lib():
    from dqsim_bosonic_b200 import build as b

    b.build()
    from dqsim_bosonic_b200 import _native

    return _native.lib()


@pytest.fixture(scope="session")
def gpu(engine_lib):
    from dqsim_bosonic_b200 import _native

    if _native.device_count() < 1:
        pytest.fail("a CUDA device is required for tests marked gpu")
    return 0


@pytest.fixture(autouse=True)
def _oracle_threads():
    import _oracle

    _oracle.set_threads(int(os.environ.get("DQSIM_ORACLE_THREADS", "1")))
    yield
    _oracle.set_threads(1)
