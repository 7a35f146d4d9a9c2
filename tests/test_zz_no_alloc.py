"""qp_pmove_static: the re-bin that runs on a fixed device array instead of
allocated scratch, checked through the C ABI against qp_species_pmove.

The caller's particle buffers are torch CUDA tensors (the caller allocates its
inputs and outputs; the entry point allocates nothing).  Two calls in a row
on different inputs must both agree with the allocating entry point bit for
bit, which also checks that the second call does not see the first call's
leftover inbox contents.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOX = [[-6.0, 6.0], [-6.0, 6.0], [0.0, 10.0]]


@pytest.fixture(scope="module")
def env():
    import torch

    import qpgpu

    assert torch.cuda.is_available()
    L = qpgpu.lib()
    ctx = qpgpu.Context(6, 6, 4, BOX)
    yield torch, qpgpu, L, ctx
    ctx.close()


def _displaced(sp, seed, amp):
    """The loaded plasma with every particle moved by up to +-amp cells."""
    pp, kp = sp.get_particles()
    rng = np.random.default_rng(seed)
    for t in range(len(kp)):
        n = kp[t]
        pp[0, :n, t] += rng.uniform(-amp, amp, n).astype(np.float32)
        pp[1, :n, t] += rng.uniform(-amp, amp, n).astype(np.float32)
        pp[2, :n, t] = rng.normal(0, 1, n).astype(np.float32)
    return pp, kp


def _planes(torch, pp, cap):
    """Eight (ntiles, cap) SoA planes on the device from ppart(8, nppmx, ntiles)."""
    nt = pp.shape[2]
    out = []
    for c in range(8):
        h = np.zeros((nt, cap), dtype=np.float32)
        h[:, : pp.shape[1]] = pp[c].T
        out.append(torch.from_numpy(h).cuda())
    return out


def _ptrs(planes):
    return (C.c_void_p * 8)(*[p.data_ptr() for p in planes])


def _static_pmove(torch, L, ix, iy, pp, kp, cap_out):
    cap_in = pp.shape[1]
    pin = _planes(torch, pp, cap_in)
    cin = torch.from_numpy(np.ascontiguousarray(kp, dtype=np.int32)).cuda()
    pout = [torch.full((len(kp), cap_out), -7.0, device="cuda") for _ in range(8)]
    cout = torch.zeros(len(kp), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = L.qp_pmove_static(ix, iy, _ptrs(pin), C.c_void_p(cin.data_ptr()), cap_in,
                           _ptrs(pout), C.c_void_p(cout.data_ptr()), cap_out,
                           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, [p.cpu().numpy() for p in pout], cout.cpu().numpy()


def _check_equal(gp, gk, planes, counts):
    assert np.array_equal(counts, gk)
    assert counts.sum() > 0
    for t in range(len(gk)):
        for c in range(8):
            assert np.array_equal(planes[c][t, : gk[t]], gp[c, : gk[t], t]), (t, c)


def test_static_pmove_matches_pmove_twice(env):
    torch, qp, L, ctx = env
    sp = qp.Species2d(ctx, ppc=(2, 2), xtras=0.5)
    base_pp, base_kp = sp.get_particles()
    for seed, amp in ((11, 5.0), (12, 9.0)):
        pp, kp = _displaced(sp, seed, amp)
        cap_out = 2 * pp.shape[1]
        rc, planes, counts = _static_pmove(torch, L, 6, 6, pp, kp, cap_out)
        assert rc == 0, L.qp_ctx_last_error(None)
        # the allocating entry point on the same input
        sp.set_particles(pp, kp)
        sp.pmove()
        gp, gk = sp.get_particles(max(sp.nppmx, int(counts.max())))
        _check_equal(gp, gk, planes, counts)
        sp.set_particles(base_pp, base_kp)
    sp.close()


def test_static_pmove_rejects_and_recovers(env):
    torch, qp, L, ctx = env
    sp = qp.Species2d(ctx, ppc=(2, 2), xtras=0.5)
    pp, kp = _displaced(sp, 21, 4.0)
    # a grid with more tiles than the fixed array can serve (checked on the host)
    dummy = (C.c_void_p * 8)(*([C.c_void_p(16)] * 8))
    dummy2 = (C.c_void_p * 8)(*([C.c_void_p(32)] * 8))
    rc = L.qp_pmove_static(11, 11, dummy, C.c_void_p(16), 64, dummy2, C.c_void_p(32), 64, None)
    assert rc < 0
    assert b"static scratch" in L.qp_ctx_last_error(None)
    # an output capacity too small for the tiles: rejected with the needed size
    rc, _, _ = _static_pmove(torch, L, 6, 6, pp, kp, 8)
    assert rc < 0
    assert b"cap_out 8 too small" in L.qp_ctx_last_error(None)
    # the next call starts from a clean status and agrees with pmove
    rc, planes, counts = _static_pmove(torch, L, 6, 6, pp, kp, 2 * pp.shape[1])
    assert rc == 0, L.qp_ctx_last_error(None)
    sp.set_particles(pp, kp)
    sp.pmove()
    gp, gk = sp.get_particles(max(sp.nppmx, int(counts.max())))
    _check_equal(gp, gk, planes, counts)
    sp.close()


def test_static_pmove_rejects_inbox_overflow_and_bad_counts(env):
    """On a 1024 x 1024 grid (4096 tiles) the fixed array leaves room for 100
    movers per tile: 200 particles leaving one tile for the same neighbour are
    refused with the inbox message, and a tile count above cap_in is refused
    with the tile-count message."""
    torch, qp, L, ctx = env
    ix = iy = 10
    mx1 = (1 << ix) // 16
    nt = mx1 * mx1
    cap_in, cap_out = 256, 512
    pin = [torch.zeros((nt, cap_in), device="cuda") for _ in range(8)]
    t0 = 10 + mx1 * 10  # tile (10, 10): cells x 160..175, y 160..175
    rng = np.random.default_rng(5)
    n = 200
    pin[0][t0, :n] = torch.from_numpy(rng.uniform(176.5, 191.5, n).astype(np.float32)).cuda()
    pin[1][t0, :n] = torch.from_numpy(rng.uniform(160.5, 175.5, n).astype(np.float32)).cuda()
    counts = np.zeros(nt, dtype=np.int32)
    counts[t0] = n
    cin = torch.from_numpy(counts).cuda()
    pout = [torch.full((nt, cap_out), -7.0, device="cuda") for _ in range(8)]
    cout = torch.zeros(nt, dtype=torch.int32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    rc = L.qp_pmove_static(ix, iy, _ptrs(pin), C.c_void_p(cin.data_ptr()), cap_in, _ptrs(pout),
                           C.c_void_p(cout.data_ptr()), cap_out, stream)
    assert rc < 0
    msg = L.qp_ctx_last_error(None)
    assert b"moved into one tile" in msg and b"holds 100" in msg, msg
    # a count above the input capacity
    counts[:] = 0
    counts[7] = cap_in + 1
    cin2 = torch.from_numpy(counts).cuda()
    rc = L.qp_pmove_static(ix, iy, _ptrs(pin), C.c_void_p(cin2.data_ptr()), cap_in, _ptrs(pout),
                           C.c_void_p(cout.data_ptr()), cap_out, stream)
    assert rc < 0
    assert b"tile count lies outside" in L.qp_ctx_last_error(None)


def test_static_pmove_allocates_nothing(env):
    """After the array is placed (context creation or a first call), a call
    leaves the device's free memory unchanged."""
    torch, qp, L, ctx = env
    sp = qp.Species2d(ctx, ppc=(2, 2), xtras=0.5)
    pp, kp = _displaced(sp, 31, 3.0)
    cap_in, cap_out = pp.shape[1], 2 * pp.shape[1]
    pin = _planes(torch, pp, cap_in)
    cin = torch.from_numpy(np.ascontiguousarray(kp, dtype=np.int32)).cuda()
    pout = [torch.zeros((len(kp), cap_out), device="cuda") for _ in range(8)]
    cout = torch.zeros(len(kp), dtype=torch.int32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = (6, 6, _ptrs(pin), C.c_void_p(cin.data_ptr()), cap_in, _ptrs(pout),
            C.c_void_p(cout.data_ptr()), cap_out, stream)
    assert L.qp_pmove_static(*args) == 0, L.qp_ctx_last_error(None)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert L.qp_pmove_static(*args) == 0, L.qp_ctx_last_error(None)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert int(cout.sum().item()) == int(kp.sum())
    sp.close()
