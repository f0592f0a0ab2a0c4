"""The C++ drop-in layer (include/cufsp.hpp) used the way the reference's own tests use the
reference API: device PropFun via cudaMemcpyFromSymbol, thrust vectors, MVFun lambda (gpu)."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

EXE = Path(__file__).resolve().parent / "cpp" / "test_dropin"


def test_cpp_dropin_program(cuda, built):
    assert EXE.exists(), "tests/cpp/test_dropin is built by python -m cuda_fsp_b200.build"
    r = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok (0 failures)" in r.stdout
