import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")


@pytest.fixture(scope="session")
def built():
    """Build the library, the test-support module and the oracle once per session (no-op when fresh)."""
    from cuda_fsp_b200 import build as B
    import oracle
    out = B.build()
    if not oracle.ORACLE_SO.exists():
        oracle.build()
    return out


@pytest.fixture(scope="session")
def cuda(built):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def testmodels(built):
    """libcufsp_testmodels.so: the library device-linked with the tests' __device__ propensities."""
    import ctypes as C
    from cuda_fsp_b200 import _lib
    path = ROOT / "tests" / "support" / "libcufsp_testmodels.so"
    lib = _lib.load(path)
    lib.tm_toggle_propfn.restype = C.c_void_p
    lib.tm_nonfact_propfn.restype = C.c_void_p
    return lib


def require_ref():
    """The reference's own compiled code (oracle/_ref/libref.so, built by oracle/Makefile from the
    reference sources and shipped with the tree).  Its absence fails the test: the comparisons with
    the reference's kernels and host functions are the strongest parity evidence and must not
    vanish from a green run."""
    import oracle
    R = oracle.ref()
    if R is None:
        pytest.fail(f"{oracle.REF_SO} is missing: build it with `make -C oracle ref` where the reference "
                    "sources are present (CUFSP_REFERENCE_SRC) and ship it with the tree")
    return R
