import glob
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _openblas():
    try:
        import scipy
        cand = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "libscipy_openblas-*.so"))
        return os.path.abspath(cand[0]) if cand else None
    except Exception:
        return None


if "JFEM_ORACLE_OPENBLAS" not in os.environ and _openblas():
    os.environ["JFEM_ORACLE_OPENBLAS"] = _openblas()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle
