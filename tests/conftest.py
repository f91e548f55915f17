import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA engine)")


@pytest.fixture(scope="session")
def built():
    """Make sure the oracle and the engine library exist (builds them if missing)."""
    import oracle
    oracle.lib()
    from rustatevec_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        import subprocess
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "rustatevec_b200", "csrc")], check=True)
    return True


@pytest.fixture(scope="session")
def be64(built):
    from rustatevec_b200 import B200Backend
    b = B200Backend(0, precision="f64")
    yield b
    b.close()


@pytest.fixture(scope="session")
def be32(built):
    from rustatevec_b200 import B200Backend
    b = B200Backend(0, precision="f32")
    yield b
    b.close()
