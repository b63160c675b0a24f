import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: runs the CUDA kernels; needs a B200 (deselect with -m 'not gpu')")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    d = ROOT / "tests" / "golden"
    return {name: np.load(d / f"{name}.npz") for name in ("tensor_ops", "lie_maps", "signatures", "streams")}
