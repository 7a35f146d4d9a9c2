"""Shared test set-up.

* ``-m gpu`` tests call the engine (libqpgpu.so) through its C ABI and compare
  with the CPU oracle on the same inputs; ``-m "not gpu"`` tests check the
  oracle against known answers and the library's exported interface.
* Configs follow QuickPIC's input deck keys (simulation.box, beam.np, ...),
  scaled down so the oracle finishes in seconds.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "quickpic-opensource_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libqpgpu.so")


BOX = [[-6.0, 6.0], [-6.0, 6.0], [0.0, 10.0]]


def make_config(ind=(6, 6, 5), ppc=(2, 2), iter=2, beams=None, store3d=True):
    """A QuickPIC-style configuration (species 1 uniform plasma, beams profile 0)."""
    if beams is None:
        beams = [dict(np=[32, 32, 32], q=-1.0, m=1.0, gamma=20000.0, peak_density=2.0,
                      quiet_start=True, center=[0.0, 0.0, 2.5], sigma=[0.5, 0.5, 0.5],
                      sigma_v=[0.0, 0.0, 0.0])]
    return dict(grid=dict(ind=list(ind), box=BOX), iter=iter,
                species=dict(ppc=list(ppc), q=-1.0, m=1.0, density=1.0, xtras=0.2),
                beams=beams, store3d=store3d)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    if den == 0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / den)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle
