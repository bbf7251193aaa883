import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "libsvm-cuda_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"),
          os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def engine():
    from svmb200 import Engine
    eng = Engine()
    if not eng.available():
        pytest.fail("GPU test selected but no CUDA device is available to libsvm_b200.so")
    return eng


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    return oracle_py.Oracle()


@pytest.fixture(scope="session")
def oracle64():
    import oracle_py
    return oracle_py.Oracle(fp64=True)
