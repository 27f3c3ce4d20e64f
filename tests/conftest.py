import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: large sizes")


@pytest.fixture(scope="session")
def restate():
    from oracle.oracle import Restatement, build
    build(with_ref=False) if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")) else None
    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference build (oracle/_ref) not present")
    return Reference()


@pytest.fixture(scope="session")
def sb():
    """The product library; on a GPU test it must load and see a B200."""
    import stream_b200
    if not stream_b200.device_ok():
        raise RuntimeError("stream_b200: no compute-capability 10.0 GPU visible")
    return stream_b200
