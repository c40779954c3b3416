import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as _oracle  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); compares libsu2b "
                            "against the oracle through the C ABI")


@pytest.fixture(scope="session")
def orc():
    """The C restatement of the reference (oracle/su2_oracle.c)."""
    if not _oracle.available("orc"):
        _oracle.build("oracle")
    return _oracle.Oracle("orc")


@pytest.fixture(scope="session")
def ref():
    """The reference's own headers behind a C ABI; only where the reference was built."""
    if not _oracle.available("ref"):
        if _oracle.reference_dir():
            _oracle.build("ref")
        else:
            pytest.skip("reference harness not built here")
    return _oracle.Oracle("ref")


def _gpu_present() -> bool:
    try:
        cudart = ctypes.CDLL("libcudart.so")
    except OSError:
        try:
            from su2_b200 import _abi
            lib = _abi.load()
            ctx = ctypes.c_void_p()
            rc = lib.su2b_ctx_create(0, 2, 2, 2, 2, 4, 1.0, 1.0, 0, 0, ctypes.byref(ctx))
            if rc == 0:
                lib.su2b_ctx_destroy(ctx)
            return rc == 0
        except Exception:
            return False
    n = ctypes.c_int(0)
    return cudart.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0


@pytest.fixture(scope="session")
def gpu():
    if not _gpu_present():
        pytest.fail("no CUDA device visible for a test marked gpu")
    import su2_b200
    su2_b200.load()
    return su2_b200


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
