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


# (C struct in include/qpgpu.h, ctypes mirror in qpgpu) pairs of the boundary
STRUCTS = [("qp_grid_desc", "_GridDesc"), ("qp_species_desc", "_SpeciesDesc"),
           ("qp_beam_desc", "_BeamDesc"), ("qp_sim_desc", "_SimDesc"),
           ("qp_step_stats", "StepStats"), ("qp_scan_desc", "_ScanDesc"),
           ("qp_scan_stats", "ScanStats"), ("qp_nn_train_desc", "_TrainDesc"),
           ("qp_nn_train_stats", "TrainStats")]


def test_descriptor_layouts_match_the_header(qp, tmp_path):
    """Every descriptor's size and field offsets, as the C compiler lays them
    out from include/qpgpu.h, equal the ctypes mirror's (a drifted field would
    pass wrong values across the boundary without any error)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "qpgpu.h"', "int main(void) {"]
    for cname, pyname in STRUCTS:
        lines.append(f'  printf("{pyname} size %zu\\n", sizeof({cname}));')
        for fname, _ in getattr(qp, pyname)._fields_:
            lines.append(f'  printf("{pyname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(root, "include"), str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = {}
    for line in out.splitlines():
        name, field, val = line.split()
        got[(name, field)] = int(val)
    for _, pyname in STRUCTS:
        st = getattr(qp, pyname)
        assert got[(pyname, "size")] == C.sizeof(st), pyname
        for fname, _ in st._fields_:
            assert got[(pyname, fname)] == getattr(st, fname).offset, (pyname, fname)
