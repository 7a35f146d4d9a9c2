"""Slices replayed from captured CUDA graphs (qp_sim_desc.use_graphs).

A slice's launches are captured once per particle-buffer parity and number of
passes enqueued and replayed for every slice with the same two.  The graph
holds device pointers; before a replay the engine compares every pointer and
value the graph holds with the current ones and captures again when one
changed (a buffer grown, the two particle buffers swapped after an odd number
of slices, a replaced plane).  Graph replay must give the results of direct
launches: the whole step against the FP64 oracle, and graph against direct
runs of the same instance, which differ only by the summation order of the
L2-reduction deposits (FP32 roundoff, 1e-4 on fields over whole steps as for
any two runs)."""
import numpy as np
import pytest
from conftest import make_config, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def qp():
    import qpgpu

    return qpgpu


def _sim(qp, cfg, use_graphs, dt=0.0):
    ind = cfg["grid"]["ind"]
    c = qp.Context(ind[0], ind[1], ind[2], cfg["grid"]["box"])
    s = cfg["species"]
    sp = qp.Species2d(c, ppc=tuple(s["ppc"]), q=s["q"], m=s["m"], density=s["density"],
                      xtras=s["xtras"])
    b = cfg["beams"][0]
    bm = qp.Beam3d(c, b["np"], q=b["q"], m=b["m"], gamma=b["gamma"],
                   peak_density=b["peak_density"], quiet_start=b["quiet_start"],
                   center=b["center"], sigma=b["sigma"], sigma_v=b["sigma_v"])
    sim = qp.Simulation(c, [sp], [bm], iter=cfg["iter"], store3d=True, use_graphs=use_graphs,
                        dt=dt, tol=cfg.get("tol", 0.0), predict=cfg.get("predict", 0))
    return c, sp, bm, sim


def _close(*objs):
    for o in objs:
        o.close()


def test_graph_step_matches_oracle(qp, oracle_mod):
    """One whole 3D step (64^2 x 32 slices, 2 passes) replayed from graphs:
    the 3D fields within 1e-4 of the FP64 oracle, like direct launches."""
    O = oracle_mod
    cfg = make_config(ind=(6, 6, 5), iter=2)
    c, sp, bm, sim = _sim(qp, cfg, True)
    st = sim.step3d()
    assert st.slices == 32
    # one graph per parity (one pass count)
    assert sim.graph_captures == 2
    o64 = O.Sim(cfg, np.float64)
    o64.begin3d()
    for j in range(1, 33):
        o64.slice(j)
    be = sim.get_3d("bexyz")
    assert rel_l2(be, o64.get("bexyz").reshape(be.shape, order="F")) < 1e-4
    q3 = sim.get_3d("q3")
    assert rel_l2(q3, o64.get("q3").reshape(q3.shape, order="F")) < 1e-4
    o64.close()
    _close(sim, bm, sp, c)


def test_graph_replay_matches_direct_launches(qp):
    """Three convergence-controlled steps with the beam push (B to 1e-4, at
    most 12 passes, quadratic start): graph replay against direct launches of
    the same instance; the pass counts may differ by a few over a step where
    the FP32 residual crosses the tolerance one pass apart."""
    cfg = make_config(ind=(6, 6, 5), iter=12)
    cfg["tol"] = 1e-4
    cfg["predict"] = 2
    a = _sim(qp, cfg, True, dt=10.0)
    b = _sim(qp, cfg, False, dt=10.0)
    for step in range(3):
        sa, sb = a[3].step3d(), b[3].step3d()
        assert abs(sa.iterations - sb.iterations) <= 4, (step, sa.iterations, sb.iterations)
        assert sa.kernels > 0
        for name in ("bexyz", "bbxyz", "q3"):
            assert rel_l2(a[3].get_3d(name), b[3].get_3d(name)) < 1e-4, (step, name)
        pa, pb = a[2].get_particles(), b[2].get_particles()
        assert pa.shape == pb.shape
    caps = a[3].graph_captures
    # a graph per parity and pass count in use, at most 12 counts
    assert 2 <= caps <= 2 * 12, caps
    assert b[3].graph_captures == 0
    _close(a[3], a[2], a[1], a[0], b[3], b[2], b[1], b[0])


def test_graph_signature_follows_buffer_swaps(qp):
    """A step run as 5 + 6 + 21 slices: after the odd first call the two
    particle buffers of the species trade roles, so the graphs captured for
    both parities no longer match and are captured again (4 captures in all);
    the second call leaves the roles as they are and the third replays.  The
    result equals the same partition run with direct launches."""
    cfg = make_config(ind=(6, 6, 5), iter=2)
    out = []
    for graphs in (True, False):
        c, sp, bm, sim = _sim(qp, cfg, graphs)
        sim.begin3d()
        sim.slices(5)
        n1 = sim.graph_captures
        sim.slices(6)
        n2 = sim.graph_captures
        sim.slices(21)
        n3 = sim.graph_captures
        sim.end3d()
        if graphs:
            assert (n1, n2, n3) == (2, 4, 4), (n1, n2, n3)
        out.append({k: sim.get_3d(k) for k in ("bexyz", "bbxyz", "q3")})
        _close(sim, bm, sp, c)
    for k in out[0]:
        assert rel_l2(out[0][k], out[1][k]) < 1e-4, k


@pytest.mark.parametrize("use_graphs", [False, True], ids=["direct", "graph"])
def test_pass_loop_stops_at_iter(qp, use_graphs):
    """A tolerance no slice meets (1e-12) with at most 5 passes: every slice
    stops after 5 passes or earlier on the stall rule (which needs 8), so
    each of the 32 slices takes exactly 5 and all are counted unconverged."""
    cfg = make_config(ind=(6, 6, 5), iter=5)
    cfg["tol"] = 1e-12
    c, sp, bm, sim = _sim(qp, cfg, use_graphs)
    st = sim.step3d()
    assert st.iterations == 5 * 32, st.iterations
    assert st.unconverged == 32
    _close(sim, bm, sp, c)


def test_graph_pass_counts_match_direct(qp):
    """Graph replay runs the passes the direct launches run: per-step pass
    totals agree (within FP32 roundoff of the residual near the tolerance)
    on two 128^2 x 128 steps, the second capped from the first's record."""
    cfg = make_config(ind=(7, 7, 7), iter=16)
    cfg["tol"] = 1e-4
    res = []
    for graphs in (True, False):
        c, sp, bm, sim = _sim(qp, cfg, graphs, dt=10.0)
        st = [sim.step3d() for _ in range(2)]
        res.append(([x.iterations for x in st], [x.unconverged for x in st],
                    sim.get_3d("bexyz")))
        _close(sim, bm, sp, c)
    (ig, ug, bg), (idir, ud, bd) = res
    for a, b in zip(ig, idir):
        assert abs(a - b) <= 0.02 * b, (ig, idir)
    assert rel_l2(bg, bd) < 1e-4
