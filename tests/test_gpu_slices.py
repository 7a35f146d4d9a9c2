"""Parity at the sizes the benchmark runs.

* Single slices of the 512 x 512 medium case (32 x 32 tiles, 512-point line
  transforms) from identical inputs: the engine runs a 3D step up to slice
  j - 1 (qp_sim_begin3d, qp_sim_slices), the state it hands to slice j -- the
  tiled particles, the Fourier-space B_perp iterate epw, the extrapolated
  current cu_k and slice j's beam charge plane -- is loaded into the oracle,
  and both run slice j.  The slice's outputs (the fields stored for the slice,
  psi, epw, cu_k) are compared with the FP32 oracle (the reference's SGL
  build) and the FP64 oracle (its DBL build).  Samples lie ahead of, inside
  and behind the beam.
* The small case of the reference's CPU-runnable configuration (128 x 128 x
  128, 2 x 2 ppc, 262,144 beam particles, 2 fixed passes), one whole 3D step
  against the FP64 oracle.

Tolerances (relative L2, except B_z, which is measured against |B_perp|: in
an axisymmetric wake B_z is roundoff, and the FP32 and FP64 oracles differ by
more than 1e-3 in it; the reasons are in each test):
  * per slice, fixed 2 passes: every field <= 1e-5 against the FP32 oracle in
    and behind the beam; ahead of it, where FP32 roundoff of the plasma-ion
    charge cancellation alone moves the FP32 oracle up to a few 1e-4 from
    FP64, within 1.5x that roundoff of both;
  * per slice, passes to a relative change of 1e-4: <= 1e-4 against the FP64
    oracle, or 1.5x the FP32 oracle's own distance where that is larger;
  * whole 128^3 step: bexyz, bbxyz and the plasma charge q3 <= 1e-3 against
    the FP64 oracle (the full-step bar on moments).
"""
import numpy as np
import pytest
from conftest import BOX, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def qp():
    import qpgpu

    return qpgpu


def medium_slice_cfg(iter=2, tol=0.0, nb=(256, 256, 16)):
    """The medium case's transverse problem (512^2, 2 x 2 ppc, beam sigma_r 0.3,
    sigma_z 0.6, nb/np 4, 1% energy spread, emittance 0.01) on 64 slices."""
    return dict(grid=dict(ind=[9, 9, 6], box=BOX), iter=iter, tol=tol,
                species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                beams=[dict(np=list(nb), q=-1.0, m=1.0, gamma=20000.0, peak_density=4.0,
                            quiet_start=True, center=[0.0, 0.0, 3.0], sigma=[0.3, 0.3, 0.6],
                            sigma_v=[0.01 / 0.3, 0.01 / 0.3, 200.0])],
                store3d=True)


def _engine(qp, cfg):
    g = cfg["grid"]["ind"]
    c = qp.Context(g[0], g[1], g[2], cfg["grid"]["box"])
    s = cfg["species"]
    sp = qp.Species2d(c, ppc=tuple(s["ppc"]), q=s["q"], m=s["m"], density=s["density"],
                      xtras=s["xtras"])
    beams = [qp.Beam3d(c, b["np"], q=b["q"], m=b["m"], gamma=b["gamma"],
                       peak_density=b["peak_density"], quiet_start=b["quiet_start"],
                       center=b["center"], sigma=b["sigma"], sigma_v=b["sigma_v"])
             for b in cfg["beams"]]
    sim = qp.Simulation(c, [sp], beams, iter=cfg["iter"], store3d=True, tol=cfg.get("tol", 0.0))
    return c, sp, beams, sim


def engine_state(sim, sp, j):
    """What slice j reads from the slice before it."""
    pp, kp = sp.get_particles()
    return dict(ppart=pp, kpic=kp, epw_k=sim.get_field("epw"), cu_k=sim.get_field("cu_k"),
                qb=sim.get_plane("qb", j))


def engine_outputs(sim, j, ny):
    be, bb = sim.get_plane("bexyz", j), sim.get_plane("bbxyz", j)
    return dict(fxy=be[0:2], psit=be[2], bxy=bb[0:2], bz=bb[2],
                psi=sim.get_field("psi")[0, :, : ny + 1], epw=sim.get_field("epw"),
                cu_k=sim.get_field("cu_k"))


def oracle_outputs(o, nx, ny):
    nxv, nyp = nx + 2, 2 * ny + 1
    fxy = o.get("fxy").reshape((2, nxv, nyp), order="F")[:, :, : ny + 1]
    bxyz = o.get("bxyz").reshape((3, nxv, nyp), order="F")[:, :, : ny + 1]
    return dict(fxy=fxy, psit=o.get("psit").reshape((nxv, nyp), order="F")[:, : ny + 1],
                bxy=bxyz[0:2], bz=bxyz[2],
                psi=o.get("psi").reshape((nxv, nyp), order="F")[:, : ny + 1],
                epw=o.get("epw_k").reshape((2, ny + 1, nx + 1), order="F"),
                cu_k=o.get("cu_k").reshape((3, ny + 1, nx + 1), order="F"))


def slice_errors(qp, O, cfg, samples):
    """{j: {field: (err vs FP32 oracle, err vs FP64 oracle, FP32 vs FP64)}} for
    each sampled slice j, each run from the engine's state after slice j-1."""
    c, sp, beams, sim = _engine(qp, cfg)
    ocfg = dict(cfg, beams=[], store3d=False)
    o32, o64 = O.Sim(ocfg, np.float32), O.Sim(ocfg, np.float64)
    nx, ny = c.nx, c.ny
    out = {}
    sim.begin3d()
    for j in samples:
        if j > sim.next_slice:
            sim.slices(j - sim.next_slice)
        st = engine_state(sim, sp, j)
        sim.slices(1)
        got = engine_outputs(sim, j, ny)
        res = {}
        for o in (o32, o64):
            o.set_state(**st)
            o.slice(j)
        e32, e64 = oracle_outputs(o32, nx, ny), oracle_outputs(o64, nx, ny)
        for k in got:
            if k == "bz":
                # B_z of an axisymmetric wake is roundoff-level (the FP32 and FP64
                # oracles differ by more than 1e-3 in it): its error is measured
                # against the size of B_perp, not of itself
                def rel(a, b):
                    return float(np.linalg.norm(np.asarray(a, np.float64) - b) /
                                 np.linalg.norm(np.asarray(e64["bxy"], np.float64)))
            else:
                rel = rel_l2
            res[k] = (rel(got[k], e32[k]), rel(got[k], e64[k]), rel(e32[k], e64[k]))
        out[j] = res
    if sim.next_slice <= c.nz:
        sim.slices(c.nz - sim.next_slice + 1)
    sim.end3d()
    for x in (o32, o64):
        x.close()
    sim.close()
    for b in beams:
        b.close()
    sp.close()
    c.close()
    return out


SAMPLES = [6, 13, 19, 26, 45]  # ahead of the beam centre, at it, behind it, in the wake


def _report(errs):
    for j, r in errs.items():
        print(j, {k: tuple(f"{v:.2e}" for v in e) for k, e in r.items()})


def test_medium_slices_fixed_passes_match_fp32_oracle(qp, oracle_mod):
    """The reference's path (2 fixed passes) at 512^2: from identical inputs
    every field a slice produces is within 1e-5 of the FP32 oracle.  The
    differences are FP32 roundoff of the transforms (a radix-4 factorisation
    against the reference's radix-2) and of the deposits' summation order,
    carried through the two passes."""
    errs = slice_errors(qp, oracle_mod, medium_slice_cfg(iter=2), SAMPLES)
    _report(errs)
    for j, r in errs.items():
        for k, (e32, e64, ref) in r.items():
            # ahead of the beam the wake is a small difference of the O(1)
            # plasma and ion charges, and FP32 roundoff alone puts the FP32
            # oracle up to a few 1e-4 away from FP64 in psi and the current
            # there: the bar is then that roundoff, for the distance to the
            # FP32 oracle and to the FP64 result alike
            assert e32 <= max(1e-5, 1.5 * ref), (j, k, e32, e64, ref)
            assert e64 <= max(1e-5, 1.5 * ref), (j, k, e32, e64, ref)
    # inside the beam and behind it the fields are large: the plain 1e-5 bar
    for j in (13, 19, 26, 45):
        for k, (e32, e64, ref) in errs[j].items():
            assert e32 <= 1e-5, (j, k, e32, e64, ref)


def test_medium_slices_to_tolerance_match_fp64_oracle(qp, oracle_mod):
    """Passes to a relative change of 1e-4 (the medium benchmark's setting):
    from identical inputs the slice's fields are within 1e-4 of the FP64
    oracle's converged fields."""
    errs = slice_errors(qp, oracle_mod, medium_slice_cfg(iter=16, tol=1e-4), SAMPLES)
    _report(errs)
    for j, r in errs.items():
        for k, (e32, e64, ref) in r.items():
            # as above: ahead of the beam FP32 roundoff of the charge
            # cancellation sets the bar where it exceeds the tolerance
            assert e64 <= max(1e-4, 1.5 * ref), (j, k, e32, e64, ref)


def small_cfg():
    """The reference's CPU-runnable case: 128^2 x 128 slices over 12 x 12 x 10
    c/wp, 2 x 2 ppc, tri-Gaussian beam of 64^3 particles, sigma (0.3, 0.3, 0.5),
    nb/np 2, gamma 20000, 2 fixed passes."""
    return dict(grid=dict(ind=[7, 7, 7], box=BOX), iter=2,
                species=dict(ppc=[2, 2], q=-1.0, m=1.0, density=1.0, xtras=0.2),
                beams=[dict(np=[64, 64, 64], q=-1.0, m=1.0, gamma=20000.0, peak_density=2.0,
                            quiet_start=True, center=[0.0, 0.0, 2.5], sigma=[0.3, 0.3, 0.5],
                            sigma_v=[0.0, 0.0, 0.0])],
                store3d=True)


def test_small_case_full_step_matches_fp64_oracle(qp, oracle_mod):
    """One whole 3D step of the 128^3 case: the stored 3D fields and the
    plasma charge are within the full-step bar of 1e-3 of the FP64 oracle;
    the FP32 oracle's own distance is printed beside the engine's."""
    O = oracle_mod
    cfg = small_cfg()
    c, sp, beams, sim = _engine(qp, cfg)
    st = sim.step3d()
    assert st.slices == 128
    o32, o64 = O.Sim(cfg, np.float32), O.Sim(cfg, np.float64)
    for o in (o32, o64):
        o.begin3d()
        for j in range(1, 129):
            o.slice(j)
    for name in ("bexyz", "bbxyz", "q3"):
        got = sim.get_3d(name)
        r64 = o64.get(name).reshape(got.shape, order="F")
        r32 = o32.get(name).reshape(got.shape, order="F")
        e, eref = rel_l2(got, r64), rel_l2(r32, r64)
        print(name, f"engine {e:.2e}  fp32 oracle {eref:.2e}")
        assert e <= 1e-3, (name, e, eref)
    sim.close()
    for b in beams:
        b.close()
    sp.close()
    c.close()
