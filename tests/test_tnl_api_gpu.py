"""The TNL-shaped C++ interface as a drop-in: tests/cpp/tnl_api_test.cpp is
ordinary TNL-style code (SparseMatrix<..., Devices::Cuda, ..., Segments>,
setRowCapacities/setElement, vectorProduct, CG/BICGStab/GMRES::solve)
compiled against tnl-dev_b200/include/TNL/b2s_tnl.h and libb2sparse.so."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
BIN = ROOT / "tnl-dev_b200" / "_build" / "tnl_api_test"


def test_cpp_binary_is_built():
    assert BIN.exists(), "run __graft_entry__.build() first"


@pytest.mark.gpu
def test_tnl_cpp_interface_on_gpu():
    r = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=600)
    print(r.stdout[-3000:], r.stderr[-2000:])
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "PASSED (0 failures)" in r.stdout
