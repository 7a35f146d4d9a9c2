"""The C ABI library (no GPU): it builds for sm_100a, loads, and exports every
entry point declared in include/qpgpu.h."""
import ctypes as C
import os
import subprocess

import pytest


@pytest.fixture(scope="module")
def qp():
    import qpgpu

    if not os.path.exists(qpgpu.LIB_PATH):
        qpgpu.build()
    return qpgpu


def test_library_exports_every_declared_symbol(qp):
    L = qp.lib()
    syms = qp.exported_symbols()
    assert len(syms) > 50
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_library_has_no_cuda_runtime_dependency(qp):
    """cudart is linked statically, so the library loads wherever the driver is."""
    out = subprocess.run(["ldd", qp.LIB_PATH], capture_output=True, text=True).stdout
    assert "libcudart" not in out


def test_errors_are_reported_not_crashed(qp):
    """A bad grid is rejected with a message before any device call."""
    L = qp.lib()
    with pytest.raises(qp.QPError, match="grid exponents"):
        qp.Context(2, 2, 2, [[-1, 1], [-1, 1], [0, 1]])
    assert b"grid exponents" in L.qp_ctx_last_error(None)


def test_oracle_is_not_linked_by_the_product(qp):
    out = subprocess.run(["ldd", qp.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in out
    nm = subprocess.run(["nm", "-D", qp.LIB_PATH], capture_output=True, text=True).stdout
    assert "oq_" not in nm
