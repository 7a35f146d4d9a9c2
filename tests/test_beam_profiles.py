"""Beam profiles 0 (with centroids and static), 1, 2, 3 and 100 (fdist3d_class.f03).

CPU tests check the oracle's loaders against known answers and statistics;
``gpu`` tests create each beam through the engine's C ABI and compare the
particles with the oracle bit for bit (both draw from ranorm's fixed seeds,
and profile 1's uniform draws from the same SplitMix64 stand-in for
RANDOM_NUMBER), and the static densities node for node.
"""
import numpy as np
import pytest

F = np.float32
BOX = [[-6.0, 6.0], [-6.0, 6.0], [0.0, 10.0]]
IND = (6, 6, 5)


def cells(box=BOX, ind=IND):
    """dx, dy, dz as init_fdist3d computes them (FP32)."""
    return tuple(F(F(box[a][1]) - F(box[a][0])) / F(1 << ind[a]) for a in range(3))


def to_cells(v, a, box=BOX, ind=IND):
    return F(F(F(v) - F(box[a][0])) / cells(box, ind)[a])


def centroid_cells(cx, cy, box=BOX, ind=IND):
    dx, dy, dz = cells(box, ind)
    ox = [F(F(F(cx[0]) * dz) * dz) / dx, F(F(cx[1]) * dz) / dx, F(cx[2]) / dx]
    oy = [F(F(F(cy[0]) * dz) * dz) / dy, F(F(cy[1]) * dz) / dy, F(cy[2]) / dy]
    return np.array(ox, dtype=F), np.array(oy, dtype=F)


PIECE_Z = [1.0, 3.0, 5.0, 7.5]
PIECE_FZ = [0.2, 1.0, 0.5, 0.1]


# ----------------------------------------------------------------- CPU oracle

def test_piecewise_table_and_charge(oracle_mod):
    O = oracle_mod
    dx, dy, dz = cells()
    nz = 1 << IND[2]
    zf, sumz = O.dist3d_001_zf(PIECE_Z, PIECE_FZ, BOX[2][0], dz, nz)
    # trapezoid integral of fz over z
    assert sumz == pytest.approx(np.trapezoid(PIECE_FZ, PIECE_Z), rel=1e-6)
    zc = (np.array(PIECE_Z) - BOX[2][0]) / float(dz)
    want = np.interp(np.arange(1, nz + 1), zc, PIECE_FZ, left=0.0, right=0.0)
    want[np.arange(1, nz + 1) >= zc[-1]] = 0.0
    assert np.allclose(zf, want, rtol=1e-5, atol=1e-6)
    with pytest.raises(AssertionError):
        O.dist3d_001_zf([1.0, 1.0], [1.0, 1.0], 0.0, dz, nz)


def test_random_loader_centroid_offsets(oracle_mod):
    """PRVDIST32_RANDOM shifts each quiet pair's midpoint off the axis by the
    centroid polynomial of (z - z0)."""
    O = oracle_mod
    cx, cy = centroid_cells((0.01, 0.05, 0.2), (0.0, -0.05, 0.1))
    O.ranorm_reset()
    x0, y0, z0 = 32.0, 32.0, 8.0
    part = O.beam_load(F(-0.01), (0, 0, 0), 20000.0, (8, 8, 16), IND, (4.0, 4.0, 3.0),
                       (x0, y0, z0), quiet=True, cx=cx, cy=cy)
    # ranorm again from the same seeds without the offsets
    O.ranorm_reset()
    base = O.beam_load(F(-0.01), (0, 0, 0), 20000.0, (8, 8, 16), IND, (4.0, 4.0, 3.0),
                       (x0, y0, z0), quiet=True)
    assert part.shape == base.shape
    dzz = part[2] - F(z0)
    offx = -(cx[0] * (dzz * dzz)) - cx[1] * dzz - cx[2]
    offy = -(cy[0] * (dzz * dzz)) - cy[1] * dzz - cy[2]
    assert np.allclose(part[0] - base[0], offx, atol=2e-5)
    assert np.allclose(part[1] - base[1], offy, atol=2e-5)


def test_ran_pfl_follows_the_longitudinal_profile(oracle_mod):
    O = oracle_mod
    dx, dy, dz = cells()
    nz = 1 << IND[2]
    zf, _ = O.dist3d_001_zf(PIECE_Z, PIECE_FZ, BOX[2][0], dz, nz)
    O.ranorm_reset()
    part = O.beam_load_pfl(F(-0.01), (32.0, 32.0, 8.0), (4.0, 4.0), (0.0, 0.0, 0.0), 20000.0,
                           (0, 0, 0), (0, 0, 0), (16, 16, 64), (64, 64, nz), zf, quiet=True)
    z = part[2]
    assert z.size > 10000 and np.all((z > 0) & (z < nz - 1))
    # density of z along the piecewise-linear dp (interpolated at z + 1, 1-based)
    h, edges = np.histogram(z, bins=nz - 1, range=(0, nz - 1))
    mid = 0.5 * (edges[:-1] + edges[1:])
    dens = np.interp(mid + 1.0, np.arange(1, nz + 1), np.abs(zf))
    dens = dens / dens.sum() * z.size
    ok = dens > 200
    assert np.all(np.abs(h[ok] - dens[ok]) < 5 * np.sqrt(dens[ok]) + 0.02 * dens[ok])
    # quiet pairs mirror x, y about the centre
    assert np.allclose(part[0, 0::2] + part[0, 1::2], 64.0, atol=1e-4)


def test_twiss_loader_correlation_and_cut(oracle_mod):
    """PRVDIST32_TWISS: the normalised transverse draws lie inside the circle
    of radius 3, and the slope of px on x is -gamma alpha / beta."""
    O = oracle_mod
    gamma, alpha = 20000.0, (0.8, -0.4)
    beta, emit = (F(200.0), F(150.0)), (F(25.0), F(30.0))
    O.ranorm_reset()
    part = O.beam_load_twiss(F(-0.01), alpha, beta, emit, 3.0, 100.0, gamma, (16, 16, 32),
                             (64, 64, 32), (32.0, 32.0, 16.0), quiet=True)
    sigx = np.sqrt(F(beta[0] * emit[0] / F(gamma)))
    sigy = np.sqrt(F(beta[1] * emit[1] / F(gamma)))
    u, v = (part[0] - 32.0) / sigx, (part[1] - 32.0) / sigy
    assert np.all(u * u + v * v <= 9.0 + 1e-3)
    for a, (sig, al, be) in enumerate(((sigx, alpha[0], beta[0]), (sigy, alpha[1], beta[1]))):
        x = part[a] - 32.0
        slope = np.sum(x * part[3 + a]) / np.sum(x * x)
        assert slope == pytest.approx(-gamma * al / be, rel=0.05)
    assert np.all(np.abs(part[5] - gamma) < 6 * 100.0)


def test_ring_loader_weights(oracle_mod):
    O = oracle_mod
    ppc = (2, 2, 2)
    bc = np.array([32.0, 32.0, 16.0], dtype=F)
    lb = np.array([20.0, 20.0, 10.0], dtype=F)
    ub = np.array([44.0, 44.0, 22.0], dtype=F)
    r1, r2 = F(8.0), F(2.0)
    qm = F(F(F(F(-1.0) / F(1.0)) / F(2)) / F(2)) / F(2)
    n = 24 * 24 * 12 * 8
    part = O.beam_load_ring(ppc, qm, 2.0, 20000.0, bc, lb, ub, r1, r2, (64, 64, 32), n)
    assert part.shape[1] == n
    tx, ty, tz = part[0], part[1], part[2]
    assert tx.min() == pytest.approx(19.25) and tx.max() == pytest.approx(42.75)
    a1 = np.abs(tz - bc[2])
    a2 = np.sqrt((tx - bc[0]) * (tx - bc[0]) + (ty - bc[1]) * (ty - bc[1]))
    a3 = np.abs(a2 - r1)
    a4 = a1 * a1 + a3 * a3
    want = F(qm * F(2.0)) * np.exp(-(a4 / F(r2 * r2) * F(0.5))).astype(F)
    assert np.allclose(part[6], want, rtol=2e-7, atol=0)
    assert np.all(part[5] == F(20000.0)) and np.all(part[3:5] == 0)


def test_file_loader_reads_and_cuts(oracle_mod, tmp_path):
    O = oracle_mod
    dx, dy, dz = cells()
    cwp = F(F(F(5.32150254) * F(1e9)) / np.sqrt(F(1e16)))
    rng = np.random.default_rng(3)
    n = 60
    rows = np.stack([-rng.uniform(-1, 11, n) * cwp, rng.uniform(-7, 7, n) * cwp,
                     rng.uniform(-7, 7, n) * cwp, rng.uniform(1e4, 2e4, n),
                     rng.normal(0, 1, n), rng.normal(0, 1, n), rng.uniform(-1, -0.5, n)], 1)
    path = tmp_path / "beam.txt"
    path.write_text("".join(" ".join(f"{v:.9g}" for v in r) + "\n" for r in rows))
    x0, y0 = to_cells(0.0, 0), to_cells(0.0, 1)
    part = O.beam_load_file(path, n, x0, y0, dx, dy, dz, cwp, (64, 64, 32), npmax=n)
    vals = np.array([[F(float(f"{v:.9g}")) for v in r] for r in rows], dtype=F)
    tx = vals[:, 1] / cwp / dx + x0
    ty = vals[:, 2] / cwp / dy + y0
    tz = -(vals[:, 0] / cwp / dz)
    keep = (tx >= 1) & (tx <= 63) & (ty >= 0) & (ty < 64) & (tz >= 0) & (tz < 32)
    assert 0 < keep.sum() < n
    assert np.array_equal(part[0], tx[keep]) and np.array_equal(part[2], tz[keep])
    assert np.array_equal(part[5], vals[keep, 3]) and np.array_equal(part[6], vals[keep, 6])


def test_static_density_is_the_analytic_profile(oracle_mod):
    O = oracle_mod
    cx, cy = centroid_cells((0.01, 0.05, 0.2), (0.0, -0.05, 0.1))
    n3 = (64, 64, 32)
    q3 = O.beam_static(F(-2.0), (32.0, 30.0, 12.0), (4.0, 5.0, 3.0), cx, cy, None, n3)
    k, i, j = 9, 20, 40
    zval = F(k) - F(12.0)
    cx0 = -(cx[0] * (zval * zval)) - cx[1] * zval - cx[2]
    cy0 = -(cy[0] * (zval * zval)) - cy[1] * zval - cy[2]
    t1 = F(-2.0) * np.exp(-(zval * zval / F(2.0) / F(9.0)))
    d = F(i) - F(32.0) + cx0
    t2 = t1 * np.exp(-(d * d / F(2.0) / F(16.0)))
    e = F(j) - F(30.0) + cy0
    want = t2 * np.exp(-(e * e / F(2.0) / F(25.0)))
    assert q3[i, j, k] == pytest.approx(float(want), rel=1e-6)
    assert np.all(q3[64:, :, :] == 0) and np.all(q3[:, 64, :] == 0) and np.all(q3[:, :, 32] == 0)
    assert q3.min() < 0 and q3.max() <= 0


# ------------------------------------------------------------- GPU parity

@pytest.fixture(scope="module")
def qp():
    import qpgpu

    return qpgpu


def _ctx(qp):
    return qp.Context(IND[0], IND[1], IND[2], BOX)


@pytest.mark.gpu
def test_profile0_centroid_beam_matches_oracle(qp, oracle_mod):
    O = oracle_mod
    c = _ctx(qp)
    kw = dict(q=-1.0, m=1.0, gamma=20000.0, peak_density=2.0, quiet_start=True,
              center=(0.5, -0.5, 2.5), sigma=(0.5, 0.6, 0.4), sigma_v=(0.1, 0.1, 100.0))
    bm = qp.Beam3d(c, (16, 16, 16), centroid_x=(0.01, 0.05, 0.2), centroid_y=(0.0, -0.05, 0.1),
                   **kw)
    got = bm.get_particles()
    qm = O.beam_qm(-1.0, 2.0, kw["sigma"], [b[0] for b in BOX], [b[1] for b in BOX], *IND,
                   16, 16, 16)
    dx, dy, dz = cells()
    sig = (F(F(0.5) / dx), F(F(0.6) / dy), F(F(0.4) / dz))
    cen = tuple(to_cells(kw["center"][a], a) for a in range(3))
    cx, cy = centroid_cells((0.01, 0.05, 0.2), (0.0, -0.05, 0.1))
    O.ranorm_reset()
    ref = O.beam_load(qm, (0.1, 0.1, 100.0), 20000.0, (16, 16, 16), IND, sig, cen, quiet=True,
                      npmax=16 * 16 * 16 + 8, cx=cx, cy=cy)
    assert got.shape == ref.shape and np.array_equal(got, ref)
    bm.close()
    c.close()


@pytest.mark.gpu
def test_profile1_piecewise_beam_matches_oracle(qp, oracle_mod):
    O = oracle_mod
    c = _ctx(qp)
    bm = qp.Beam3d(c, (16, 16, 32), profile=1, q=-1.0, peak_density=2.0, gamma=20000.0,
                   center=(0.0, 0.5, 0.0), sigma=(0.5, 0.4, 0.0), sigma_v=(0.1, 0.2, 100.0),
                   centroid_x=(0.0, 0.02, 0.1), piecewise_z=PIECE_Z, piecewise_fz=PIECE_FZ)
    got = bm.get_particles()
    dx, dy, dz = cells()
    nz = 1 << IND[2]
    zf, sumz = O.dist3d_001_zf(PIECE_Z, PIECE_FZ, BOX[2][0], dz, nz)
    qm = O.beam_qm2(-1.0, 2.0, 1.0, 0.5, 0.4, sumz, dx, dy, dz, 16, 16, 32)
    cx, cy = centroid_cells((0.0, 0.02, 0.1), (0.0, 0.0, 0.0))
    O.ranorm_reset()
    ref = O.beam_load_pfl(qm, (to_cells(0.0, 0), to_cells(0.5, 1), to_cells(0.0, 2)),
                          (F(F(0.5) / dx), F(F(0.4) / dy)), (0.1, 0.2, 100.0), 20000.0, cx, cy,
                          (16, 16, 32), (64, 64, nz), zf, quiet=True)
    assert got.shape == ref.shape and np.array_equal(got, ref)
    bm.close()
    c.close()


@pytest.mark.gpu
def test_profile2_twiss_beam_matches_oracle(qp, oracle_mod):
    O = oracle_mod
    c = _ctx(qp)
    alpha, beta, emit = (0.8, -0.4), (500.0, 400.0), (10.0, 12.5)
    bm = qp.Beam3d(c, (16, 16, 16), profile=2, q=-1.0, peak_density=2.0, gamma=20000.0,
                   center=(0.0, 0.0, 3.0), alpha=alpha, beta=beta, emittance=emit, sigmaz=0.5,
                   sigma_vz=200.0)
    got = bm.get_particles()
    dx, dy, dz = cells()
    sx = np.sqrt(F(F(F(beta[0]) * F(emit[0])) / F(20000.0)))
    sy = np.sqrt(F(F(F(beta[1]) * F(emit[1])) / F(20000.0)))
    qm = O.beam_qm2(-1.0, 2.0, 1.5, sx, sy, 0.5, dx, dy, dz, 16, 16, 16)
    O.ranorm_reset()
    ref = O.beam_load_twiss(qm, alpha, (F(F(beta[0]) / dx), F(F(beta[1]) / dy)),
                            (F(F(emit[0]) / dx), F(F(emit[1]) / dy)), F(F(0.5) / dz), 200.0,
                            20000.0, (16, 16, 16), (64, 64, 32),
                            tuple(to_cells(v, a) for a, v in enumerate((0.0, 0.0, 3.0))))
    assert got.shape == ref.shape and np.array_equal(got, ref)
    bm.close()
    c.close()


@pytest.mark.gpu
def test_profile3_file_beam_matches_oracle(qp, oracle_mod, tmp_path):
    O = oracle_mod
    cwp = F(F(F(5.32150254) * F(1e9)) / np.sqrt(F(1e16)))
    rng = np.random.default_rng(5)
    n = 200
    rows = np.stack([-rng.uniform(-1, 11, n) * cwp, rng.uniform(-7, 7, n) * cwp,
                     rng.uniform(-7, 7, n) * cwp, rng.uniform(1e4, 2e4, n),
                     rng.normal(0, 1, n), rng.normal(0, 1, n), rng.uniform(-1, -0.5, n)], 1)
    path = tmp_path / "beam.txt"
    path.write_text("".join(" ".join(f"{v:.9g}" for v in r) + "\n" for r in rows))
    c = _ctx(qp)
    bm = qp.Beam3d(c, n, profile=3, file_name=path, n0=1e16, center=(0.5, -0.25, 0.0))
    got = bm.get_particles()
    dx, dy, dz = cells()
    ref = O.beam_load_file(path, n, to_cells(0.5, 0), to_cells(-0.25, 1), dx, dy, dz, cwp,
                           (64, 64, 32), npmax=n)
    assert 0 < got.shape[1] < n
    assert got.shape == ref.shape and np.array_equal(got, ref)
    bm.close()
    c.close()


@pytest.mark.gpu
def test_profile100_ring_beam_matches_oracle(qp, oracle_mod):
    O = oracle_mod
    c = _ctx(qp)
    bm = qp.Beam3d(c, (1, 1, 1), profile=100, q=-1.0, peak_density=2.0, gamma=20000.0,
                   center=(0.0, 0.0, 4.0), ppc=(2, 2, 2), range_x=(-3.0, 3.0),
                   range_y=(-3.0, 3.0), range_z=(2.0, 6.0), r1=1.5, r2=0.5)
    got = bm.get_particles()
    dx, dy, dz = cells()
    lb = [to_cells(v, a) for a, v in enumerate((-3.0, -3.0, 2.0))]
    ub = [to_cells(v, a) for a, v in enumerate((3.0, 3.0, 6.0))]
    bc = [to_cells(v, a) for a, v in enumerate((0.0, 0.0, 4.0))]
    qm = F(F(F(F(-1.0) / F(1.0)) / F(2)) / F(2)) / F(2)
    ref = O.beam_load_ring((2, 2, 2), qm, 2.0, 20000.0, bc, lb, ub, F(F(1.5) / dx),
                           F(F(0.5) / dx), (64, 64, 32), 64 * 64 * 32 * 8)
    assert got.shape == ref.shape and np.array_equal(got, ref)
    bm.close()
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("profile", [0, 1])
def test_static_beam_density_matches_oracle(qp, oracle_mod, profile):
    O = oracle_mod
    c = _ctx(qp)
    kw = dict(q=-1.0, peak_density=2.0, gamma=20000.0, center=(0.3, -0.2, 4.0),
              sigma=(0.5, 0.6, 0.7), centroid_x=(0.01, 0.05, 0.2), centroid_y=(0.0, -0.05, 0.1),
              static=True)
    if profile == 1:
        kw.update(piecewise_z=PIECE_Z, piecewise_fz=PIECE_FZ)
    bm = qp.Beam3d(c, (16, 16, 16), profile=profile, **kw)
    assert bm.np() == 0
    got = bm.get_q3d()
    dx, dy, dz = cells()
    nz = 1 << IND[2]
    if profile == 0:
        qm = O.beam_qm(-1.0, 2.0, kw["sigma"], [b[0] for b in BOX], [b[1] for b in BOX], *IND,
                       16, 16, 16)
        zf = None
    else:
        zf, sumz = O.dist3d_001_zf(PIECE_Z, PIECE_FZ, BOX[2][0], dz, nz)
        qm = O.beam_qm2(-1.0, 2.0, 1.0, 0.5, 0.6, sumz, dx, dy, dz, 16, 16, 16)
    amp = F(F(F(2.0) * F(qm)) / abs(F(qm)))
    cx, cy = centroid_cells(kw["centroid_x"], kw["centroid_y"])
    sig = (F(F(0.5) / dx), F(F(0.6) / dy), F(F(0.7) / dz))
    cen = tuple(to_cells(kw["center"][a], a) for a in range(3))
    ref = O.beam_static(amp, cen, sig, cx, cy, zf, (64, 64, nz))
    assert np.array_equal(got, ref)
    # a static beam is not deposited again by qdp
    bm.qdp()
    assert np.array_equal(bm.get_q3d(), ref)
    bm.close()
    c.close()


@pytest.mark.gpu
def test_frozen_and_static_beams_in_a_step(qp):
    """evolution = false leaves a beam's particles where they are at the push
    (push_beam3d); a static beam keeps its density through the step and still
    drives the plasma."""
    c = _ctx(qp)
    sp = qp.Species2d(c, ppc=(2, 2), q=-1.0, m=1.0, density=1.0, xtras=0.2)
    kw = dict(q=-1.0, m=1.0, gamma=200.0, peak_density=1.0, center=(0.0, 0.0, 2.5),
              sigma=(0.5, 0.5, 0.5), sigma_v=(0.0, 0.0, 0.0))
    moving = qp.Beam3d(c, (8, 8, 8), **kw)
    frozen = qp.Beam3d(c, (8, 8, 8), evolution=False, **kw)
    static = qp.Beam3d(c, (8, 8, 8), static=True, **dict(kw, center=(1.0, 0.0, 6.0)))
    p_moving, p_frozen = moving.get_particles(), frozen.get_particles()
    q_static = static.get_q3d()
    sim = qp.Simulation(c, [sp], [moving, frozen, static], iter=2, store3d=True, dt=5.0)
    sim.step3d()
    assert not np.array_equal(moving.get_particles(), p_moving)
    assert np.array_equal(frozen.get_particles(), p_frozen)
    assert np.array_equal(static.get_q3d(), q_static)
    sim.close()
    for b in (moving, frozen, static):
        b.close()
    sp.close()
    c.close()


@pytest.mark.gpu
def test_beam_profile_edge_cases(qp, tmp_path):
    """Beams that miss the box load no particles; bad descriptors are errors,
    not faults."""
    c = _ctx(qp)
    # profile 1 whose piecewise z range lies behind the box: npp = 0 (dist3d_001)
    b1 = qp.Beam3d(c, (8, 8, 8), profile=1, piecewise_z=[20.0, 30.0],
                   piecewise_fz=[1.0, 1.0], sigma=(0.5, 0.5, 0.0))
    assert b1.np() == 0
    b1.qdp()
    assert not np.any(b1.get_q3d())
    b1.close()
    # ring whose y range misses the box: no particles (dist3d_100)
    b2 = qp.Beam3d(c, (1, 1, 1), profile=100, ppc=(1, 1, 1), range_x=(-3.0, 3.0),
                   range_y=(20.0, 30.0), range_z=(1.0, 2.0), r1=1.0, r2=0.5)
    assert b2.np() == 0
    b2.close()
    # errors: unknown profile, non-increasing piecewise z, missing file, static profile 2
    with pytest.raises(qp.QPError, match="profile must be"):
        qp.Beam3d(c, (8, 8, 8), profile=4)
    with pytest.raises(qp.QPError, match="monotonically"):
        qp.Beam3d(c, (8, 8, 8), profile=1, piecewise_z=[2.0, 1.0], piecewise_fz=[1.0, 1.0])
    with pytest.raises(qp.QPError, match="cannot open"):
        qp.Beam3d(c, 10, profile=3, file_name=tmp_path / "missing.txt", n0=1e16)
    with pytest.raises(qp.QPError, match="static"):
        qp.Beam3d(c, (8, 8, 8), profile=2, static=True, alpha=(0, 0), beta=(1, 1),
                  emittance=(1, 1))
    # a short file is an error
    short = tmp_path / "short.txt"
    short.write_text("-100 0 0 20000 0 0 -1\n")
    with pytest.raises(qp.QPError, match="read beam file"):
        qp.Beam3d(c, 3, profile=3, file_name=short, n0=1e16)
    # commas and Fortran d exponents read like blanks and e
    ok = tmp_path / "fortran.txt"
    ok.write_text("-1.0d2, 0.0, 0.0, 2.0D4, 0.0, 0.0, -1.0\n")
    b3 = qp.Beam3d(c, 1, profile=3, file_name=ok, n0=1e16)
    p = b3.get_particles()
    assert p.shape == (7, 1) and p[5, 0] == np.float32(2.0e4) and p[6, 0] == np.float32(-1.0)
    b3.close()
    c.close()


@pytest.mark.gpu
def test_beam_restart_round_trip(qp, tmp_path):
    """beam3d%wrst / %rrst in the reference's RST/Beam-NNNN layout: a beam
    written after a pushed step and read back into another beam has the same
    particles, bit for bit; a step from either gives the same fields."""
    box = [[-6.0, 6.0], [-6.0, 6.0], [0.0, 10.0]]
    c = qp.Context(6, 6, 5, box)
    sp = qp.Species2d(c, ppc=(2, 2))
    b1 = qp.Beam3d(c, [16, 16, 16], q=-1.0, m=1.0, gamma=20000.0, peak_density=2.0,
                   quiet_start=True, center=[0.0, 0.0, 2.5], sigma=[0.5, 0.5, 0.5],
                   sigma_v=[0.1, 0.1, 10.0])
    sim = qp.Simulation(c, [sp], [b1], iter=2, store3d=True, dt=10.0)
    sim.step3d()
    b1.write_restart(str(tmp_path), beam=1, rank=0, step=3)
    f = tmp_path / "RST" / "Beam-0001" / "RST-beam0001-0000000000_00000003.qprst"
    assert f.exists()
    raw = f.read_bytes()
    assert raw[:8] == b"QPRST001"
    tp = int(np.frombuffer(raw[8:16], dtype=np.int64)[0])
    assert tp == b1.np()
    b2 = qp.Beam3d(c, [16, 16, 16], q=-1.0, m=1.0, gamma=20000.0, peak_density=1.0,
                   quiet_start=True, center=[0.0, 0.0, 4.0], sigma=[0.3, 0.3, 0.3])
    b2.read_restart(str(tmp_path), beam=1, rank=0, step=3)
    assert np.array_equal(b2.get_particles(), b1.get_particles())
    with pytest.raises(qp.QPError, match="cannot open"):
        b2.read_restart(str(tmp_path), beam=2, rank=0, step=3)
    for b in (b1, b2):
        b.close()
    sim.close()
    sp.close()
    c.close()
