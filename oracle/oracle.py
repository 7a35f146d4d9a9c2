"""ctypes front end of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the B200 engine.  Only tests/,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module.  PARITY UNPINNED: the reference (QuickPIC-OpenSource, Fortran) has no
tests or golden vectors and cannot be compiled here; the restatement is pinned
by the known-answer tests under tests/golden/.

Arrays use the reference's Fortran layouts (see qp_oracle.h) and are passed as
numpy arrays in Fortran order, e.g. a real-space field of dimension ``dim`` is
``np.zeros((dim, nx + 2, 2 * ny + 1), order="F")``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.oq_ranorm.restype = C.c_double
        for s in ("f", "d"):
            getattr(_lib, f"oq_sim_create_{s}").restype = C.c_void_p
            getattr(_lib, f"oq_sim_size_{s}").restype = C.c_longlong
            for n in ("destroy", "step3d", "begin3d", "slice", "get", "size"):
                getattr(_lib, f"oq_sim_{n}_{s}").argtypes = None
    return _lib


def _sfx(dtype) -> str:
    return "f" if np.dtype(dtype) == np.float32 else "d"


def _ctype(dtype):
    return C.c_float if np.dtype(dtype) == np.float32 else C.c_double


def _p(a: np.ndarray):
    # every multi-dimensional array is a Fortran-layout reference array
    if a.ndim > 1 and not a.flags["F_CONTIGUOUS"]:
        raise ValueError("oracle arrays must be Fortran-contiguous (reference layout)")
    if not a.flags["F_CONTIGUOUS"]:
        raise ValueError("oracle arrays must be contiguous")
    return a.ctypes.data_as(C.c_void_p)


def _call(name, dtype, *args):
    fn = getattr(lib(), f"{name}_{_sfx(dtype)}")
    ct = _ctype(dtype)
    cargs = []
    for a in args:
        if isinstance(a, np.ndarray):
            cargs.append(_p(a))
        elif isinstance(a, float):
            cargs.append(ct(a))
        elif isinstance(a, (int, np.integer)):
            cargs.append(C.c_int(int(a)))
        else:
            cargs.append(a)
    rc = fn(*cargs)
    return rc


# ----------------------------------------------------------------- layouts
def rs_zeros(dim, indx, indy, dtype=np.float32):
    nx, ny = 1 << indx, 1 << indy
    return np.zeros((dim, nx + 2, 2 * ny + 1), dtype=dtype, order="F")


def ks_zeros(dim, indx, indy, dtype=np.float32):
    nx, ny = 1 << indx, 1 << indy
    return np.zeros((dim, ny + 1, nx + 1), dtype=dtype, order="F")


def ffc(indx, indy, dtype=np.float32, ax=0.912871, ay=0.912871, affp=1.0):
    nx, ny = 1 << indx, 1 << indy
    t = np.zeros((2, ny, nx), dtype=dtype, order="F")
    _call("oq_ffc", dtype, t, indx, indy, float(ax), float(ay), float(affp))
    return t


# --------------------------------------------------------------- transforms
def fftrk(rs, ks, kind, indx, indy):
    rc = _call("oq_fftrk", rs.dtype, rs, ks, rs.shape[0], kind, indx, indy)
    assert rc == 0, rc


def fftkr(rs, ks, kind, indx, indy):
    rc = _call("oq_fftkr", rs.dtype, rs, ks, rs.shape[0], kind, indx, indy)
    assert rc == 0, rc


def line(v, parity, xpass, isign, indx, indy):
    """One NR pass on a contiguous line of n+2 values (in place)."""
    rc = _call("oq_line", v.dtype, v, 1, parity, xpass, isign, indx, indy)
    assert rc == 0


def pot(q, p, t, indx, indy):
    _call("oq_pot", q.dtype, q, p, t, indx, indy)


def smooth(q, qs, t, indx, indy):
    _call("oq_smooth", q.dtype, q, qs, t, indx, indy)


def elf(q, fxy, t, indx, indy):
    _call("oq_elf", q.dtype, q, fxy, t, indx, indy)


def bf(cu, bxy, t, indx, indy):
    _call("oq_bf", cu.dtype, cu, bxy, t, indx, indy)


def vpot(cu, a, t, indx, indy):
    _call("oq_vpot", cu.dtype, cu, a, t, indx, indy)


def bfqp(cu, dcu, amu, bxy, t, aa, dex, indx, indy):
    _call("oq_bfqp", cu.dtype, cu, dcu, amu, bxy, t, float(aa), float(dex), indx, indy)


def div(f, df, indx, indy):
    _call("oq_div", f.dtype, f, df, f.shape[0], indx, indy)


def grad(df, f, indx, indy):
    _call("oq_grad", df.dtype, df, f, indx, indy)


def cguard(rs, indx, indy):
    _call("oq_cguard", rs.dtype, rs, rs.shape[0], indx, indy)


def acguard(rs, indx, indy):
    _call("oq_acguard", rs.dtype, rs, rs.shape[0], indx, indy)


# ---------------------------------------------------------------- particles
def ntiles(indx, indy):
    nx, ny = 1 << indx, 1 << indy
    return ((nx - 1) // 16 + 1) * ((ny - 1) // 16 + 1)


def dist2d_000(indx, indy, xppc, yppc, q=-1.0, den=1.0, dtype=np.float32):
    nx, ny = 1 << indx, 1 << indy
    npmax = xppc * yppc * nx * ny
    part = np.zeros((8, npmax), dtype=dtype, order="F")
    npp = C.c_int(0)
    rc = _call("oq_dist2d_000", dtype, part, npmax, C.byref(npp), xppc, yppc, float(q),
               float(den), indx, indy)
    assert rc == 0
    return part[:, : npp.value].copy(order="F")


def dist2d_prof(indx, indy, box, xppc, yppc, profile, q=-1.0, den=1.0, center=(0.0, 0.0),
                inner_radius=(0.0, 0.0), outer_radius=(0.0, 0.0), radius=0.0, width=0.0,
                r=(), fr=(), s=0.0, long_s=(), long_fs=(), dtype=np.float32):
    """The profile-10/11/12 (and 0) loaders with a piecewise longitudinal factor."""
    nx, ny = 1 << indx, 1 << indy
    npmax = xppc * yppc * nx * ny
    pr = np.array([profile, xppc, yppc, q, den, box[0][0], box[0][1], box[1][0], box[1][1],
                   indx, indy, center[0], center[1], inner_radius[0], inner_radius[1],
                   outer_radius[0], outer_radius[1], radius, width, s, len(r), len(long_s)]
                  + list(r) + list(fr) + list(long_s) + list(long_fs), dtype=dtype)
    part = np.zeros((8, npmax), dtype=dtype, order="F")
    npp = C.c_int(0)
    rc = _call("oq_dist2d_prof", dtype, part, npmax, C.byref(npp), pr)
    assert rc == 0, rc
    return part[:, : npp.value].copy(order="F")


def bin_particles(part, indx, indy, xtras=0.2, nppmx0=None):
    """PPDBLKP2L + PPPMOVIN2L: linear part(8, n) -> (ppart, kpic, nppmx0)."""
    dtype = part.dtype
    nt = ntiles(indx, indy)
    kpic = np.zeros(nt, dtype=np.int32)
    nppmx = C.c_int(0)
    rc = _call("oq_ppdblkp2l", dtype, part, kpic, part.shape[1], C.byref(nppmx), indx, indy)
    assert rc == 0, rc
    if nppmx0 is None:
        nppmx0 = int((1.0 + xtras) * nppmx.value)
    ppart = np.zeros((8, nppmx0, nt), dtype=dtype, order="F")
    rc = _call("oq_pppmovin2l", dtype, part, ppart, kpic, part.shape[1], nppmx0, indx, indy)
    assert rc == 0, rc
    return ppart, kpic, nppmx0


def check_tiles(ppart, kpic, indx, indy):
    return _call("oq_pppcheck2l", ppart.dtype, ppart, kpic, ppart.shape[1], indx, indy)


def qdeposit(ppart, kpic, q, indx, indy):
    _call("oq_ppgppost2l", ppart.dtype, ppart, q, kpic, ppart.shape[1], indx, indy)


def extpsi(ppart, kpic, psi, qbm, dex, indx, indy):
    _call("oq_wpgpsipost2l_qp", ppart.dtype, ppart, psi, kpic, float(qbm), ppart.shape[1],
          indx, indy, float(dex))


def amjdp(ppart, kpic, fxy, bxy, psit, cu, dcu, amu, qbm, dt, dex, indx, indy):
    _call("oq_ppgrdcjppost2l_qp", ppart.dtype, ppart, fxy, bxy, psit, cu, dcu, amu, kpic,
          float(qbm), float(dt), 1.0, ppart.shape[1], indx, indy, float(dex))


def push(ppart, kpic, fxy, bxy, psit, qbm, dt, dex, indx, indy):
    """PPGRBPPUSHF23L_QP; returns (ncl, ihole, ntmax)."""
    nt = ntiles(indx, indy)
    ntmax = ppart.shape[1]
    ncl = np.zeros((8, nt), dtype=np.int32, order="F")
    ihole = np.zeros((2, ntmax + 1, nt), dtype=np.int32, order="F")
    rc = _call("oq_ppgrbppushf23l_qp", ppart.dtype, ppart, fxy, bxy, psit, kpic, ncl, ihole,
               float(qbm), float(dt), 1.0, ppart.shape[1], ntmax, indx, indy, float(dex))
    assert rc == 0, rc
    return ncl, ihole, ntmax


def pmove(ppart, kpic, ncl, ihole, ntmax, indx, indy):
    return _call("oq_pmove", ppart.dtype, ppart, kpic, ncl, ihole, ppart.shape[1], ntmax,
                 indx, indy)


# ------------------------------------------------------------------- beams
def ranorm_reset():
    lib().oq_ranorm_reset()


def ranorm():
    return lib().oq_ranorm()


def beam_qm(q, peak, sig, lo, hi, indx, indy, indz, npx, npy, npz, dtype=np.float32):
    out = np.zeros(1, dtype=dtype)
    _call("oq_beam_qm", dtype, float(q), float(peak), np.asarray(sig, dtype=dtype),
          np.asarray(lo, dtype=dtype), np.asarray(hi, dtype=dtype), indx, indy, indz, npx,
          npy, npz, out)
    return float(out[0])


def beam_load(qm, sigv, gamma, np3, ind3, sig_cells, center_cells, quiet=True,
              npmax=None, cx=(0, 0, 0), cy=(0, 0, 0), dtype=np.float32):
    """PRVDIST32_RANDOM from the fixed ranorm seeds (caller resets ranorm); cx, cy
    are the centroid polynomials in cells."""
    npx, npy, npz = np3
    if npmax is None:
        npmax = npx * npy * npz + 2
    part = np.zeros((7, npmax), dtype=dtype, order="F")
    npp = C.c_int(0)
    rc = _call("oq_prvdist32_random", dtype, part, npmax, C.byref(npp), float(qm),
               float(sigv[0]), float(sigv[1]), float(sigv[2]), float(gamma), npx, npy, npz,
               ind3[0], ind3[1], ind3[2], float(sig_cells[0]), float(sig_cells[1]),
               float(sig_cells[2]), float(center_cells[0]), float(center_cells[1]),
               float(center_cells[2]), np.asarray(cx, dtype=dtype),
               np.asarray(cy, dtype=dtype), 1 if quiet else 0)
    assert rc == 0, rc
    return part[:, : npp.value].copy(order="F")


def dist3d_001_zf(z, fz, zmin, dz, nz, dtype=np.float32):
    """init_fdist3d_001's sumz and dist3d_001's slice table zf(1:nz)."""
    zz = np.ascontiguousarray(z, dtype=dtype)
    ff = np.ascontiguousarray(fz, dtype=dtype)
    zf = np.zeros(nz, dtype=dtype)
    sumz = np.zeros(1, dtype=dtype)
    rc = _call("oq_dist3d_001_zf", dtype, zz, ff, zz.size, float(zmin), float(dz), nz, zf, sumz)
    assert rc == 0, "piecewise_z is not increasing"
    return zf, float(sumz[0])


def beam_qm2(q, peak, e, sx, sy, sz, dx, dy, dz, npx, npy, npz, dtype=np.float32):
    """Charge per particle of beam profiles 1 (e = 1, sz = sumz) and 2 (e = 1.5)."""
    out = np.zeros(1, dtype=dtype)
    _call("oq_beam_qm2", dtype, float(q), float(peak), float(e), float(sx), float(sy), float(sz),
          float(dx), float(dy), float(dz), npx, npy, npz, out)
    return float(out[0])


def beam_load_pfl(qm, center_cells, sig_cells, sigv, gamma, cx, cy, np3, n3, dp, quiet=True,
                  seed=0x5eed, npmax=None, dtype=np.float32):
    """PRVDIST32_RAN_PFL (caller resets ranorm); dp = the slice profile zf(1:nz)."""
    npx, npy, npz = np3
    if npmax is None:
        npmax = npx * npy * npz + 8
    part = np.zeros((7, npmax), dtype=dtype, order="F")
    npp = C.c_int(0)
    d = np.array(dp, dtype=dtype)
    rc = _call("oq_prvdist32_ran_pfl", dtype, part, npmax, C.byref(npp), float(qm),
               float(center_cells[0]), float(center_cells[1]), float(center_cells[2]),
               float(sig_cells[0]), float(sig_cells[1]), float(sigv[0]), float(sigv[1]),
               float(sigv[2]), float(gamma), np.asarray(cx, dtype=dtype),
               np.asarray(cy, dtype=dtype), npx, npy, npz, n3[0], n3[1], n3[2], d,
               1 if quiet else 0, C.c_ulonglong(seed))
    assert rc == 0, rc
    return part[:, : npp.value].copy(order="F")


def beam_load_twiss(qm, alpha, beta_cells, emit_cells, sigz_cells, sigvz, gamma, np3, n3,
                    center_cells, quiet=True, npmax=None, dtype=np.float32):
    """PRVDIST32_TWISS (caller resets ranorm)."""
    npx, npy, npz = np3
    if npmax is None:
        npmax = npx * npy * npz + 8
    part = np.zeros((7, npmax), dtype=dtype, order="F")
    npp = C.c_int(0)
    rc = _call("oq_prvdist32_twiss", dtype, part, npmax, C.byref(npp), float(qm),
               np.asarray(alpha, dtype=dtype), np.asarray(beta_cells, dtype=dtype),
               np.asarray(emit_cells, dtype=dtype), float(sigz_cells), float(gamma),
               float(sigvz), npx, npy, npz, n3[0], n3[1], n3[2], float(center_cells[0]),
               float(center_cells[1]), float(center_cells[2]), 1 if quiet else 0)
    assert rc == 0, rc
    return part[:, : npp.value].copy(order="F")


def beam_load_file(path, npt, x0, y0, dx, dy, dz, cwp, n3, npmax=None, dtype=np.float32):
    """dist3d_003: particles read from a text file."""
    if npmax is None:
        npmax = max(npt, 1)
    part = np.zeros((7, npmax), dtype=dtype, order="F")
    npp = C.c_int(0)
    rc = _call("oq_dist3d_003", dtype, str(path).encode(), npt, part, npmax, C.byref(npp),
               float(x0), float(y0), float(dx), float(dy), float(dz), float(cwp), n3[0], n3[1],
               n3[2])
    assert rc == 0, rc
    return part[:, : npp.value].copy(order="F")


def beam_load_ring(ppc, qm, amp, gamma, bc, lb, ub, r1, r2, n3, npmax, dtype=np.float32):
    """dist3d_100: a ring on a lattice of ppc particles per cell."""
    part = np.zeros((7, npmax), dtype=dtype, order="F")
    npp = C.c_int(0)
    rc = _call("oq_dist3d_100", dtype, part, npmax, C.byref(npp),
               np.asarray(ppc, dtype=np.int32), float(qm), float(amp), float(gamma),
               np.asarray(bc, dtype=dtype), np.asarray(lb, dtype=dtype),
               np.asarray(ub, dtype=dtype), float(r1), float(r2), n3[0], n3[1], n3[2])
    assert rc == 0, rc
    return part[:, : npp.value].copy(order="F")


def beam_static(amp, center_cells, sig_cells, cx, cy, zf, n3, dtype=np.float32):
    """Static-beam density of dist3d_000 (zf None) or dist3d_001 as q3(nx+2, ny+1, nz+1)."""
    nx, ny, nz = n3
    q3 = np.zeros((nx + 2, ny + 1, nz + 1), dtype=dtype, order="F")
    zp = None if zf is None else np.ascontiguousarray(zf, dtype=dtype)
    _call("oq_beam_static", dtype, float(amp), float(center_cells[0]), float(center_cells[1]),
          float(center_cells[2]), float(sig_cells[0]), float(sig_cells[1]),
          float(sig_cells[2]), np.asarray(cx, dtype=dtype), np.asarray(cy, dtype=dtype),
          zp if zp is not None else C.c_void_p(0), nx, ny, nz, q3)
    return q3


def beam_deposit(part, ind3, dtype=np.float32):
    nx, ny, nz = (1 << i for i in ind3)
    q3 = np.zeros((nx + 2, ny + 1, nz + 1), dtype=dtype, order="F")
    _call("oq_pgpost32l", dtype, part, part.shape[1], q3, ind3[0], ind3[1], ind3[2])
    return q3


def beam_push(part, fxyz, bxyz, qbm, dt, dex, dxi, ind3, dtype=np.float32):
    """PGBPUSH32L_QP on part(7, np) with 3D fields (3, nx+2, ny+1, nz+1); returns the
    pushed particles, (7, np_new), after conducting-boundary drops."""
    p = np.array(part, dtype=dtype, order="F", copy=True)
    fe = np.asfortranarray(fxyz, dtype=dtype)
    fb = np.asfortranarray(bxyz, dtype=dtype)
    n = _call("oq_pgbpush32l_qp", dtype, p, p.shape[1], fe, fb, float(qbm), float(dt),
              float(dex), float(dxi), ind3[0], ind3[1], ind3[2])
    return p[:, :n]


# -------------------------------------------------------------- simulation
P_FIXED = 22
B_NPAR = 18
W = dict(psi=1, fxy=2, bxyz=3, psit=4, cu=5, dcu=6, amu=7, epw_k=8, cu_k=9, qe=10, qb=11,
         epwb_k=12, ppart=13, kpic=14, bexyz=15, bbxyz=16, q3=17, q3d=18, qn=19, beam0=20,
         nppmx=21, dcu_k=22, bxyz_k=23, np=24, qsp=25, passes=26, unconverged=27, vpot3d=28, epw_b2=29,
         epw_b3=30)


def sim_params(cfg) -> np.ndarray:
    """Pack a config dict (see tests/conftest.py: small_config) for oq_sim_create."""
    g = cfg["grid"]
    sp = cfg["species"]
    p = np.zeros(P_FIXED + B_NPAR * len(cfg["beams"]), dtype=np.float64)
    p[0:3] = g["ind"]
    p[3:9] = [g["box"][0][0], g["box"][0][1], g["box"][1][0], g["box"][1][1], g["box"][2][0],
              g["box"][2][1]]
    p[9] = cfg["iter"]
    p[10:12] = sp["ppc"]
    p[12] = sp["q"]
    p[13] = sp["m"]
    p[14] = sp["density"]
    p[15] = sp.get("xtras", 0.2)
    p[16] = len(cfg["beams"])
    p[17] = 1 if cfg.get("store3d", True) else 0
    p[18] = cfg.get("dt", 0.0)  # 3D time step; > 0 pushes the beams after the slices
    p[19] = cfg.get("tol", 0.0)  # > 0: B passes per slice until |d epw| <= tol |epw|
    p[20] = 1 if cfg.get("vpot", False) else 0  # keep the 3D vector potential
    p[21] = int(cfg.get("predict", 0))  # B start: 1 linear, 2 quadratic extrapolation
    for b, bm in enumerate(cfg["beams"]):
        o = P_FIXED + B_NPAR * b
        p[o:o + 3] = bm["np"]
        p[o + 3] = bm["q"]
        p[o + 4] = bm["m"]
        p[o + 5] = bm["gamma"]
        p[o + 6] = bm["peak_density"]
        p[o + 7] = 1 if bm.get("quiet_start", True) else 0
        p[o + 8:o + 11] = bm["center"]
        p[o + 11:o + 14] = bm["sigma"]
        p[o + 14:o + 17] = bm["sigma_v"]
        p[o + 17] = bm.get("npmax", int(np.prod(bm["np"])) + 8)
    return p


class Sim:
    """The oracle's restatement of go_simulation for one rank and one stage."""

    def __init__(self, cfg, dtype=np.float32):
        self.dtype = np.dtype(dtype)
        self.s = _sfx(dtype)
        p = sim_params(cfg).astype(self.dtype)
        L = lib()
        fn = getattr(L, f"oq_sim_create_{self.s}")
        fn.restype = C.c_void_p
        self.h = fn(_p(p), C.c_int(len(p)))
        assert self.h, "oracle sim_create failed"
        self.cfg = cfg

    def _f(self, n):
        return getattr(lib(), f"oq_sim_{n}_{self.s}")

    def begin3d(self):
        rc = self._f("begin3d")(C.c_void_p(self.h))
        assert rc == 0, rc

    def slice(self, j):
        rc = self._f("slice")(C.c_void_p(self.h), C.c_int(j))
        assert rc == 0, rc

    def step3d(self):
        rc = self._f("step3d")(C.c_void_p(self.h))
        assert rc == 0, rc

    def get(self, what):
        w = W[what]
        fn = self._f("size")
        fn.restype = C.c_longlong
        n = fn(C.c_void_p(self.h), C.c_int(w))
        assert n >= 0
        out = np.zeros(max(n, 1), dtype=self.dtype)
        rc = self._f("get")(C.c_void_p(self.h), C.c_int(w), _p(out), C.c_longlong(n))
        assert rc == 0, rc
        return out[:n]

    def set(self, what, arr):
        """Set part of the state one slice hands to the next: "ppart"
        (8, nppmx, ntiles), "kpic", "epw_k", "cu_k", "epw_b2"/"epw_b3" (the
        predictor's earlier B_perp) or "qb" (the next slice's beam charge
        plane, used once)."""
        a = np.asfortranarray(arr, dtype=self.dtype).ravel(order="F")
        rc = self._f("set")(C.c_void_p(self.h), C.c_int(W[what]), _p(a), C.c_longlong(a.size))
        assert rc == 0, (what, rc)

    def set_state(self, ppart, kpic, epw_k, cu_k, qb=None):
        """The whole state a slice reads from the slice before it: tiled
        particles ppart(8, nppmx, ntiles) and kpic, the Fourier-space B_perp
        iterate and extrapolated current, and the beam charge plane of the
        next slice (nx+2, ny+1) or (nx+2, 2ny+1)."""
        self.set("ppart", ppart)
        self.set("kpic", np.asarray(kpic, dtype=np.float64))
        self.set("epw_k", epw_k)
        self.set("cu_k", cu_k)
        if qb is not None:
            full = np.zeros((qb.shape[0], 2 * self.ny + 1), dtype=np.float64, order="F")
            full[:, : qb.shape[1]] = qb
            self.set("qb", full)

    @property
    def ny(self):
        return 1 << int(self.cfg["grid"]["ind"][1])

    def close(self):
        if self.h:
            self._f("destroy")(C.c_void_p(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
