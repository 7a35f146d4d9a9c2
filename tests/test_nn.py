"""The learned start of the B passes: its tensor-core kernels against the CPU
restatement of the network (oracle/nn_oracle.py), its recording and training
on the GPU, and what the trained network gains over the starts without it.

Tolerances: the engine rounds inputs, weights, activations and the output
gradient to bfloat16 and accumulates in FP32 (tcgen05); the oracle rounds at
the same places and accumulates in float64.  A different summation order can
move a value across a bfloat16 rounding boundary, so the forward pass is
compared at 5e-3 and the gradients at 3e-2 (relative L2, per layer)."""
import numpy as np
import pytest
from conftest import BOX, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def qp():
    import qpgpu

    return qpgpu


@pytest.fixture(scope="module")
def N():
    import nn_oracle

    return nn_oracle


def _params(N, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    p = []
    for ci, co in zip(N.CIN, N.COUT):
        p.append(rng.normal(0, scale * np.sqrt(2.0 / (9 * ci)), 9 * ci * co))
        p.append(rng.normal(0, 0.05, co))
    p = np.concatenate(p).astype(np.float32)
    # the padding outputs of layer 5 stay zero, as in the engine
    o = sum(N.layer_sizes()[:4])
    w5 = p[o:o + 9 * 32 * 16].reshape(9, 32, 16)
    w5[:, :, 2:] = 0.0
    p[o + 9 * 32 * 16 + 2:] = 0.0
    return p


@pytest.mark.parametrize("shape", [(2, 6, 128), (1, 3, 256)])
def test_forward_matches_oracle(qp, N, shape):
    nb, h, w = shape
    net = qp.Predictor(seed=1)
    p = _params(N, 5)
    net.set_params(p)
    assert np.array_equal(net.get_params(), p)
    rng = np.random.default_rng(6)
    x = rng.normal(0, 1, (nb, 16, h, w)).astype(np.float32)
    got = net.forward(x)
    exp, _, _ = N.forward(p, x)
    assert got.shape == exp.shape
    assert rel_l2(got, exp) < 5e-3, rel_l2(got, exp)
    net.close()


def test_loss_gradient_matches_oracle(qp, N):
    """Loss and the gradient of every layer's weights and biases, from the
    forward, data-gradient and weight-gradient kernels, against the oracle."""
    net = qp.Predictor(seed=1)
    p = _params(N, 7)
    net.set_params(p)
    rng = np.random.default_rng(8)
    x = rng.normal(0, 1, (2, 16, 5, 128)).astype(np.float32)
    t = rng.normal(0, 1, (2, 2, 5, 128)).astype(np.float32)
    loss, g = net.loss_grad(x, t)
    eloss, eg = N.loss_grad(p, x, t)
    assert abs(loss - eloss) < 1e-3 * eloss
    o = 0
    for l, (ci, co) in enumerate(zip(N.CIN, N.COUT)):
        nw = 9 * ci * co
        gw, ew = g[o:o + nw], eg[o:o + nw]
        gb, eb = g[o + nw:o + nw + co], eg[o + nw:o + nw + co]
        assert rel_l2(gw, ew) < 3e-2, (l, rel_l2(gw, ew))
        assert rel_l2(gb, eb) < 3e-2, (l, rel_l2(gb, eb))
        o += nw + co
    net.close()


def _sim(qp, ind, peak, sigma_r, tol=1e-4, iter=16, predict=0, seed_center=2.5,
         use_graphs=False):
    c = qp.Context(ind[0], ind[1], ind[2], BOX)
    sp = qp.Species2d(c, ppc=(2, 2))
    bm = qp.Beam3d(c, [64, 64, 64], q=-1.0, m=1.0, gamma=20000.0, peak_density=peak,
                   quiet_start=True, center=[0.0, 0.0, seed_center],
                   sigma=[sigma_r, sigma_r, 0.5], sigma_v=[0.0, 0.0, 0.0])
    sim = qp.Simulation(c, [sp], [bm], iter=iter, store3d=True, tol=tol, predict=predict,
                        use_graphs=use_graphs)
    return c, sp, bm, sim


def _close(*objs):
    for o in objs:
        o.close()


def test_recording_and_training(qp):
    """One 3D step records one pair per slice; the coordinate channels are the
    mode coordinates; training on the pairs lowers the loss."""
    c, sp, bm, sim = _sim(qp, (7, 7, 5), 2.0, 0.3)
    data = qp.TrainingSet(64)
    sim.record(data)
    sim.step3d()
    assert len(data) == 32
    img, tgt, sc = data.get(20)
    kx = np.arange(128)[:, None] / 128.0
    ky = np.arange(128)[None, :] / 128.0
    assert np.abs(img[9] - kx).max() < 4e-3 and np.abs(img[10] - ky).max() < 4e-3
    assert np.abs(img[11] - (10.0 / 32) * 25.6).max() < 2e-2  # the slice width
    assert np.all(img[12:] == 0)
    assert sc > 0 and np.isfinite(tgt).all()
    net = qp.Predictor(seed=3)
    st = net.train(data, steps=300, batch=8, lr=2e-3, seed=1)
    assert st.last_loss < 0.7 * st.first_loss, (st.first_loss, st.last_loss)
    _close(net, data, sim, bm, sp, c)


def test_learned_start_needs_fewer_passes(qp):
    """Train the network on slices of four beams (128^2, 128 slices, passes to
    a relative change of 1e-4, the carried start as the reference has it), then
    run a held-out beam from the carried start, the linear and quadratic
    extrapolations and the learned start: the learned start needs fewer passes
    than the carried one, and the converged fields agree to the tolerance."""
    data = qp.TrainingSet(4 * 128)
    for peak, sr in ((1.0, 0.25), (3.0, 0.35), (6.0, 0.2), (2.0, 0.45)):
        c, sp, bm, sim = _sim(qp, (7, 7, 7), peak, sr)
        sim.record(data)
        sim.step3d()
        _close(sim, bm, sp, c)
    net = qp.Predictor(seed=11)
    st = net.train(data, steps=2000, batch=16, lr=1e-3, seed=2)
    res = {}
    for predict in (0, 1, 2, 3):
        c, sp, bm, sim = _sim(qp, (7, 7, 7), 4.0, 0.3, predict=predict)
        if predict == 3:
            sim.set_predictor(net)
        s = sim.step3d()
        res[predict] = (s.iterations, s.unconverged, sim.get_3d("bexyz"), sim.get_3d("bbxyz"))
        _close(sim, bm, sp, c)
    print("passes: carried", res[0][0], "linear", res[1][0], "quadratic", res[2][0],
          "learned", res[3][0],
          "loss", st.first_loss, "->", st.last_loss, "train ms", st.gpu_ms)
    assert res[3][0] < res[0][0]
    for k in (2, 3):
        assert rel_l2(res[3][k], res[0][k]) < 1e-3
    # the learned start replayed from CUDA graphs (the network's launches
    # captured with the slice) gives the same passes and fields
    c, sp, bm, sim = _sim(qp, (7, 7, 7), 4.0, 0.3, predict=3, use_graphs=True)
    sim.set_predictor(net)
    s = sim.step3d()
    assert sim.graph_captures >= 2
    assert abs(s.iterations - res[3][0]) <= 0.02 * res[3][0], (s.iterations, res[3][0])
    for k, name in ((2, "bexyz"), (3, "bbxyz")):
        assert rel_l2(sim.get_3d(name), res[3][k]) < 1e-3
    _close(sim, bm, sp, c)
    _close(net, data)
