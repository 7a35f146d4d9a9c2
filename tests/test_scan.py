"""The batched parameter scan (qp_scan_run / qp_scan_tune).

Instances of different grid sizes stepped concurrently by the scan must end
where the same instances end when stepped one by one (up to the atomic-order
roundoff of the deposits, 1e-4 on fields as for whole steps), and the scan
must count every instance's particle-slices.
"""
import numpy as np
import pytest
from conftest import make_config, rel_l2

SIZES = [(6, 6, 4), (5, 5, 4), (6, 6, 5), (5, 5, 5)]


@pytest.fixture(scope="module")
def qp():
    import qpgpu

    return qpgpu


def _instance(qp, ind, peak):
    cfg = make_config(ind=ind)
    b = cfg["beams"][0]
    c = qp.Context(ind[0], ind[1], ind[2], cfg["grid"]["box"])
    s = cfg["species"]
    sp = qp.Species2d(c, ppc=tuple(s["ppc"]), q=s["q"], m=s["m"], density=s["density"],
                      xtras=s["xtras"])
    bm = qp.Beam3d(c, [16, 16, 16], q=b["q"], m=b["m"], gamma=b["gamma"], peak_density=peak,
                   quiet_start=True, center=b["center"], sigma=b["sigma"], sigma_v=b["sigma_v"])
    sim = qp.Simulation(c, [sp], [bm], iter=2, store3d=True, dt=0.0)
    return c, sp, bm, sim


def _close(insts):
    for c, sp, bm, sim in insts:
        sim.close()
        bm.close()
        sp.close()
        c.close()


@pytest.mark.gpu
def test_scan_matches_instances_stepped_alone(qp):
    peaks = [1.0, 2.0, 4.0, 0.5]
    a = [_instance(qp, ind, p) for ind, p in zip(SIZES, peaks)]
    b = [_instance(qp, ind, p) for ind, p in zip(SIZES, peaks)]
    st = qp.scan_run([i[3] for i in a], steps=2, workers=4)
    assert st.failed == 0 and st.workers == 4 and st.gpu_ms > 0
    want = sum(i[1].np() * i[0].nz * 2 for i in a)
    assert st.particle_slices == want
    for i in b:
        i[3].step3d()
        i[3].step3d()
    for x, y in zip(a, b):
        for name in ("psi", "bxyz"):
            fa, fb = x[3].get_field(name), y[3].get_field(name)
            assert rel_l2(fa, fb) < 1e-4, name
        la, lb = x[3].lineout(3), y[3].lineout(3)
        assert rel_l2(la, lb) < 1e-4
    _close(a + b)


@pytest.mark.gpu
def test_scan_tune_and_sequential_workers(qp):
    insts = [_instance(qp, ind, 2.0) for ind in SIZES[:3]]
    sims = [i[3] for i in insts]
    w, rate = qp.scan_tune(sims, probe_steps=1)
    assert w in (1, 2, 3) and rate > 0
    st = qp.scan_run(sims, steps=1, workers=1)
    assert st.workers == 1 and st.failed == 0
    _close(insts)


@pytest.mark.gpu
def test_scan_refuses_shared_contexts(qp):
    c, sp, bm, sim = _instance(qp, SIZES[1], 1.0)
    sim2 = qp.Simulation(c, [sp], [bm], iter=2, store3d=True, dt=0.0)
    with pytest.raises(qp.QPError, match="share a context"):
        qp.scan_run([sim, sim2], steps=1)
    sim2.close()
    _close([(c, sp, bm, sim)])


@pytest.mark.parametrize("n", [16, 64])
def test_scan_instances_follow_the_stated_distribution(n):
    """bench.py's scan instances (host logic, no GPU): seeded, grids among
    128^2 / 256^2 / 512^2 with 256 slices, nb/np and sigma_r in their ranges
    with (nb/np) sigma_r^2 <= 1, beam particles growing with the grid."""
    import bench

    a, b = bench.scan_instances(n), bench.scan_instances(n)
    assert a == b
    seen = set()
    for cfg in a:
        ind = cfg["grid"]["ind"]
        assert ind[0] == ind[1] and ind[0] in (7, 8, 9) and ind[2] == 8
        seen.add(ind[0])
        bm = cfg["beams"][0]
        peak, sr = bm["peak_density"], bm["sigma"][0]
        assert 0.5 <= peak <= 20.0 and 0.1 <= sr <= 0.5 and peak * sr * sr <= 1.0
        assert bm["sigma"][2] == 0.5
        nb = int(np.prod(bm["np"]))
        assert nb == {7: 262144, 8: 1048576, 9: 2097152}[ind[0]]
    assert seen == {7, 8, 9}
