import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "tests", ROOT / "ramses-cpp_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on a B200)")


@pytest.fixture(scope="session")
def oracle():
    from refsupport import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    d = ROOT / "tests" / "golden"

    def load(name):
        return np.load(d / f"{name}.npz")
    return load


@pytest.fixture(scope="session")
def reference_available():
    from refsupport import REF_SRC, ORACLE_DIR
    return REF_SRC.exists() or (ORACLE_DIR / "_ref" / "libref_harness3d.so").exists()


@pytest.fixture(scope="session")
def rgpu_lib():
    """librgpu.so, built in-tree on demand (nvcc cross-compiles without a GPU)."""
    import build as rgbuild
    import rgpu
    if not rgpu.LIB_PATH.exists():
        rgbuild.build()
    return rgpu.lib()
