"""qpgpu -- Python host side of the B200 QuickPIC slice engine.

The engine is the shared library ``libqpgpu.so`` next to this file (C ABI in
``include/qpgpu.h``).  This module binds it with ctypes and mirrors the
reference's Fortran class interface for the per-slice path, with the same
method names and argument meaning:

* :class:`Field2d`   -- ``field2d`` (fftrk/fftkr/pot/grad/div/elf/bf/bfqp/smooth,
  as/add/sub/mult, cg/ag)  (QuickPIC source/field2d_class.f03)
* :class:`Species2d` -- ``species2d`` (qdp/extpsi/amjdp/push/renew/cbq)
  (source/species2d_class.f03)
* :class:`Beam3d`    -- ``beam3d`` (qdp, qdp(q, slice))  (source/beam3d_class.f03)
* :class:`Simulation` -- the fused 3D step of ``simulation%go``
  (source/simulation_class.f03:593-769) with all state on the GPU.

Errors: a negative return code of the library raises :class:`QPError` (the
reference's ``err%equit``); capacity overflows are recovered inside the
library by growing the buffers, as ``part2d%pmove`` does.

There is no CPU fallback: importing this module without the built library, or
calling it without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqpgpu.so")

__all__ = ["QPError", "Context", "Field2d", "Species2d", "Beam3d", "Simulation", "lib",
           "build", "exported_symbols", "LIB_PATH", "Predictor", "TrainingSet"]


class QPError(RuntimeError):
    pass


_lib = None


def build() -> str:
    """Compile libqpgpu.so for sm_100a with the package Makefile."""
    import subprocess

    subprocess.run(["make", "-s", "-C", os.path.dirname(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QPError(f"{LIB_PATH} is missing: build it with `make -C "
                          f"{os.path.dirname(HERE)}` (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        L.qp_ctx_last_error.restype = C.c_char_p
        L.qp_ctx_last_need.restype = C.c_longlong
        L.qp_species_np.restype = C.c_longlong
        L.qp_beam_np.restype = C.c_longlong
        _lib = L
    return _lib


def exported_symbols():
    """Names of the qp_* functions declared in include/qpgpu.h."""
    import re

    hdr = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "qpgpu.h")
    txt = open(hdr).read()
    return sorted(set(re.findall(r"\b(qp_[a-z0-9_]+)\s*\(", txt)))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class _GridDesc(C.Structure):
    _fields_ = [("indx", C.c_int), ("indy", C.c_int), ("indz", C.c_int),
                ("box", (C.c_double * 2) * 3)]


class _SpeciesDesc(C.Structure):
    _fields_ = [("profile", C.c_int), ("ppc", C.c_int * 2), ("q", C.c_float), ("m", C.c_float),
                ("density", C.c_float), ("xtras", C.c_float), ("center", C.c_float * 2),
                ("inner_radius", C.c_float * 2), ("outer_radius", C.c_float * 2),
                ("radius", C.c_float), ("width", C.c_float),
                ("nr", C.c_int), ("r", C.POINTER(C.c_float)), ("fr", C.POINTER(C.c_float)),
                ("ns", C.c_int), ("s", C.POINTER(C.c_float)), ("fs", C.POINTER(C.c_float))]


class _BeamDesc(C.Structure):
    _fields_ = [("profile", C.c_int), ("np", C.c_int * 3), ("q", C.c_float), ("m", C.c_float),
                ("gamma", C.c_float), ("peak_density", C.c_float), ("quiet_start", C.c_int),
                ("center", C.c_float * 3), ("sigma", C.c_float * 3),
                ("sigma_v", C.c_float * 3), ("npmax", C.c_longlong),
                ("centroid_x", C.c_float * 3), ("centroid_y", C.c_float * 3),
                ("static_density", C.c_int), ("frozen", C.c_int), ("npiece", C.c_int),
                ("ppc", C.c_int * 3), ("piecewise_z", C.POINTER(C.c_float)),
                ("piecewise_fz", C.POINTER(C.c_float)), ("file_name", C.c_char_p),
                ("seed", C.c_ulonglong), ("alpha", C.c_float * 2), ("beta", C.c_float * 2),
                ("emittance", C.c_float * 2), ("n0", C.c_float), ("range_x", C.c_float * 2),
                ("range_y", C.c_float * 2), ("range_z", C.c_float * 2), ("r1", C.c_float),
                ("r2", C.c_float), ("reserved", C.c_float * 1)]


class _SimDesc(C.Structure):
    _fields_ = [("iter", C.c_int), ("store3d", C.c_int), ("use_graphs", C.c_int),
                ("dt", C.c_float), ("tol", C.c_float), ("vpot", C.c_int),
                ("predict", C.c_int), ("reserved", C.c_int * 1)]


class StepStats(C.Structure):
    _fields_ = [("slices", C.c_int), ("iterations", C.c_int), ("regrowths", C.c_int),
                ("kernels", C.c_int), ("gpu_ms", C.c_double), ("unconverged", C.c_int)]


class Context:
    """One GPU context for a grid of 2**indx x 2**indy x 2**indz cells."""

    def __init__(self, indx, indy, indz, box, device=0):
        g = _GridDesc()
        g.indx, g.indy, g.indz = indx, indy, indz
        for a in range(3):
            g.box[a][0], g.box[a][1] = box[a]
        h = C.c_void_p()
        self._L = lib()
        self._check(self._L.qp_ctx_create(C.byref(g), device, C.byref(h)), ctx=None)
        self.h = h
        self.indx, self.indy, self.indz = indx, indy, indz
        self.nx, self.ny, self.nz = 1 << indx, 1 << indy, 1 << indz
        dex, dxi = C.c_float(), C.c_float()
        self._L.qp_ctx_spacing(self.h, C.byref(dex), C.byref(dxi))
        self.dex, self.dxi = dex.value, dxi.value

    def _check(self, rc, ctx="self"):
        if rc < 0:
            c = self.h if ctx == "self" else None
            msg = self._L.qp_ctx_last_error(c)
            raise QPError(msg.decode() if msg else f"qpgpu error {rc}")
        return rc

    def sync(self):
        self._check(self._L.qp_ctx_sync(self.h))

    def timer_start(self):
        """Record a start event on the engine's stream."""
        self._check(self._L.qp_ctx_timer_start(self.h))

    def timer_stop(self):
        """Record a stop event, wait for it, return device milliseconds since start."""
        ms = C.c_double()
        self._check(self._L.qp_ctx_timer_stop(self.h, C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            self._L.qp_ctx_destroy(self.h)
            self.h = None

    # reference layouts
    def rs_shape(self, dim):
        return (dim, self.nx + 2, 2 * self.ny + 1)

    def ks_shape(self, dim):
        return (dim, self.ny + 1, self.nx + 1)


class Field2d:
    """field2d: a real-space / Fourier-space pair with the reference's state flag."""

    def __init__(self, ctx: Context, dim, state=0):
        self.ctx, self.dim = ctx, dim
        h = C.c_void_p()
        ctx._check(ctx._L.qp_field2d_create(ctx.h, dim, state, C.byref(h)))
        self.h = h

    @property
    def state(self):
        return self.ctx._L.qp_field2d_state(self.h)

    def _c(self, rc):
        return self.ctx._check(rc)

    # data movement
    def set_rs(self, a):
        a = np.asfortranarray(a, dtype=np.float32).reshape(self.ctx.rs_shape(self.dim), order="F")
        self._c(self.ctx._L.qp_field2d_upload_rs(self.h, _ptr(a)))

    def get_rs(self):
        out = np.zeros(self.ctx.rs_shape(self.dim), dtype=np.float32, order="F")
        self._c(self.ctx._L.qp_field2d_download_rs(self.h, _ptr(out)))
        return out

    def set_ks(self, a):
        a = np.asfortranarray(a, dtype=np.float32).reshape(self.ctx.ks_shape(self.dim), order="F")
        self._c(self.ctx._L.qp_field2d_upload_ks(self.h, _ptr(a)))

    def get_ks(self):
        out = np.zeros(self.ctx.ks_shape(self.dim), dtype=np.float32, order="F")
        self._c(self.ctx._L.qp_field2d_download_ks(self.h, _ptr(out)))
        return out

    # field2d methods
    def fftrk(self, kind):
        self._c(self.ctx._L.qp_field2d_fftrk(self.h, kind))

    def fftkr(self, kind):
        self._c(self.ctx._L.qp_field2d_fftkr(self.h, kind))

    def pot(self, that):
        self._c(self.ctx._L.qp_field2d_pot(self.h, that.h))

    def smooth(self, that):
        self._c(self.ctx._L.qp_field2d_smooth(self.h, that.h))

    def elf(self, that):
        self._c(self.ctx._L.qp_field2d_elf(self.h, that.h))

    def bf(self, that):
        self._c(self.ctx._L.qp_field2d_bf(self.h, that.h))

    def vpot(self, that):
        self._c(self.ctx._L.qp_field2d_vpot(self.h, that.h))

    def div(self, that):
        self._c(self.ctx._L.qp_field2d_div(self.h, that.h))

    def grad(self, that):
        self._c(self.ctx._L.qp_field2d_grad(self.h, that.h))

    def bfqp(self, dcu, amu, bxy, c, dex):
        self._c(self.ctx._L.qp_field2d_bfqp(self.h, dcu.h, amu.h, bxy.h, C.c_float(c),
                                            C.c_float(dex)))

    def as_(self, value):
        self._c(self.ctx._L.qp_field2d_as(self.h, C.c_float(value)))

    def copy_from(self, that):
        self._c(self.ctx._L.qp_field2d_copy(self.h, that.h))

    def add(self, a1, a2, dim=None, dim1=None, dim2=None):
        if dim is None:
            self._c(self.ctx._L.qp_field2d_add(self.h, a1.h, a2.h))
        else:
            d, d1, d2 = (np.asarray(v, dtype=np.int32) for v in (dim, dim1, dim2))
            self._c(self.ctx._L.qp_field2d_add_comp(self.h, a1.h, a2.h, _ptr(d), _ptr(d1),
                                                    _ptr(d2), len(d)))

    def sub(self, a1, a2, dim=None, dim1=None, dim2=None):
        if dim is None:
            self._c(self.ctx._L.qp_field2d_sub(self.h, a1.h, a2.h))
        else:
            d, d1, d2 = (np.asarray(v, dtype=np.int32) for v in (dim, dim1, dim2))
            self._c(self.ctx._L.qp_field2d_sub_comp(self.h, a1.h, a2.h, _ptr(d), _ptr(d1),
                                                    _ptr(d2), len(d)))

    def mult(self, a1, value, dim=None, dim1=None):
        if dim is None:
            self._c(self.ctx._L.qp_field2d_mult(self.h, a1.h, C.c_float(value)))
        else:
            d, d1 = (np.asarray(v, dtype=np.int32) for v in (dim, dim1))
            v = np.asarray(value, dtype=np.float32)
            self._c(self.ctx._L.qp_field2d_mult_comp(self.h, a1.h, _ptr(d), _ptr(d1), _ptr(v),
                                                     len(d)))

    def cg(self):
        self._c(self.ctx._L.qp_field2d_cg(self.h))

    def ag(self):
        self._c(self.ctx._L.qp_field2d_ag(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.ctx._L.qp_field2d_destroy(self.h)
            self.h = None


class Species2d:
    """species2d: plasma of profile 0 (uniform), 10 (elliptic hollow channel: center,
    inner_radius, outer_radius), 11 (Gaussian ring: center, radius, width) or 12
    (tabulated radial density: center, r, fr), optionally scaled by a
    piecewise-linear longitudinal density (long_s, long_fs) at propagation
    distance s.  Lengths are in the units of the box."""

    def __init__(self, ctx: Context, ppc=(2, 2), q=-1.0, m=1.0, density=1.0, xtras=0.2, s=0.0,
                 profile=0, center=(0.0, 0.0), inner_radius=(0.0, 0.0),
                 outer_radius=(0.0, 0.0), radius=0.0, width=0.0, r=None, fr=None,
                 long_s=None, long_fs=None):
        d = _SpeciesDesc()
        d.profile = profile
        d.ppc[0], d.ppc[1] = ppc
        d.q, d.m, d.density, d.xtras = q, m, density, xtras
        d.center[0], d.center[1] = center
        d.inner_radius[0], d.inner_radius[1] = inner_radius
        d.outer_radius[0], d.outer_radius[1] = outer_radius
        d.radius, d.width = radius, width
        keep = []  # the arrays must live through the create call

        def arr(v):
            a = np.ascontiguousarray(v, dtype=np.float32)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_float)), len(a)

        if r is not None:
            d.r, d.nr = arr(r)
            d.fr, _ = arr(fr)
        if long_s is not None:
            d.s, d.ns = arr(long_s)
            d.fs, _ = arr(long_fs)
        h = C.c_void_p()
        ctx._check(ctx._L.qp_species_create(ctx.h, C.byref(d), C.c_float(s), C.byref(h)))
        self.ctx, self.h = ctx, h
        self.qbm = q / m
        self.dt = ctx.dxi

    def _c(self, rc):
        return self.ctx._check(rc)

    @property
    def ntiles(self):
        return self.ctx._L.qp_species_ntiles(self.h)

    @property
    def nppmx(self):
        return self.ctx._L.qp_species_nppmx(self.h)

    def np(self):
        return int(self.ctx._L.qp_species_np(self.h))

    def qdp(self, qe):
        self._c(self.ctx._L.qp_species_qdp(self.h, qe.h))

    def extpsi(self, psi, dex):
        self._c(self.ctx._L.qp_species_extpsi(self.h, psi.h, C.c_float(dex)))

    def amjdp(self, fxy, bxyz, psit, cu, amu, dcu, dex):
        self._c(self.ctx._L.qp_species_amjdp(self.h, fxy.h, bxyz.h, psit.h, cu.h, amu.h, dcu.h,
                                             C.c_float(dex)))

    def push(self, fxy, bxyz, psit, dex):
        self._c(self.ctx._L.qp_species_push(self.h, fxy.h, bxyz.h, psit.h, C.c_float(dex)))

    def partpush(self, fxy, bxyz, psit, dex):
        self._c(self.ctx._L.qp_species_partpush(self.h, fxy.h, bxyz.h, psit.h, C.c_float(dex)))

    def pmove(self):
        self._c(self.ctx._L.qp_species_pmove(self.h))

    def renew(self, s=0.0):
        self._c(self.ctx._L.qp_species_renew(self.h, C.c_float(s)))

    def cbq(self, pos):
        self._c(self.ctx._L.qp_species_cbq(self.h, pos))

    def get_particles(self, nppmx=None):
        """(ppart(8, nppmx, ntiles), kpic(ntiles)) in the reference layout."""
        nppmx = nppmx or self.nppmx
        pp = np.zeros((8, nppmx, self.ntiles), dtype=np.float32, order="F")
        kp = np.zeros(self.ntiles, dtype=np.int32)
        self._c(self.ctx._L.qp_species_download(self.h, _ptr(pp), _ptr(kp), nppmx))
        return pp, kp

    def set_particles(self, ppart, kpic):
        pp = np.asfortranarray(ppart, dtype=np.float32)
        kp = np.ascontiguousarray(kpic, dtype=np.int32)
        self._c(self.ctx._L.qp_species_upload(self.h, _ptr(pp), _ptr(kp), pp.shape[1]))

    def get_qn(self):
        out = np.zeros(self.ctx.rs_shape(1), dtype=np.float32, order="F")
        self._c(self.ctx._L.qp_species_download_qn(self.h, _ptr(out)))
        return out

    def get_q(self):
        out = np.zeros(self.ctx.rs_shape(1), dtype=np.float32, order="F")
        self._c(self.ctx._L.qp_species_download_q(self.h, _ptr(out)))
        return out

    def get_q3(self, pos):
        out = np.zeros((self.ctx.nx + 2, self.ctx.ny + 1), dtype=np.float32, order="F")
        self._c(self.ctx._L.qp_species_download_q3(self.h, pos, _ptr(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.ctx._L.qp_species_destroy(self.h)
            self.h = None


class Beam3d:
    """beam3d with one of the fdist3d profiles: 0 tri-Gaussian, 1 Gaussian with a
    piecewise longitudinal profile, 2 Twiss parameters, 3 particles read from a
    file, 100 ring (fdist3d_class.f03).  Keys follow beam(i) of the input file;
    `np3` is np(1:3) (for profile 3 the particle count np); `static` puts the
    analytic density of profiles 0 and 1 on the grid; `evolution=False` keeps
    the beam where it is at the push."""

    def __init__(self, ctx: Context, np3, q=-1.0, m=1.0, gamma=20000.0, peak_density=1.0,
                 quiet_start=True, center=(0, 0, 0), sigma=(1, 1, 1), sigma_v=(0, 0, 0),
                 npmax=0, profile=0, centroid_x=(0, 0, 0), centroid_y=(0, 0, 0),
                 static=False, evolution=True, piecewise_z=None, piecewise_fz=None, seed=0,
                 alpha=(0, 0), beta=(0, 0), emittance=(0, 0), sigmaz=None, sigma_vz=None,
                 file_name=None, n0=0.0, range_x=(0, 0), range_y=(0, 0), range_z=(0, 0),
                 ppc=(1, 1, 1), r1=0.0, r2=0.0):
        d = _BeamDesc()
        d.profile = int(profile)
        if np.ndim(np3) == 0:
            np3 = (int(np3), 1, 1)
        sigma, sigma_v = list(sigma), list(sigma_v)
        if sigmaz is not None:
            sigma[2] = sigmaz
        if sigma_vz is not None:
            sigma_v[2] = sigma_vz
        for a in range(3):
            d.np[a] = int(np3[a])
            d.center[a], d.sigma[a], d.sigma_v[a] = center[a], sigma[a], sigma_v[a]
            d.centroid_x[a], d.centroid_y[a] = centroid_x[a], centroid_y[a]
            d.ppc[a] = int(ppc[a])
        d.q, d.m, d.gamma, d.peak_density = q, m, gamma, peak_density
        d.quiet_start = 1 if quiet_start else 0
        d.npmax = int(npmax)
        d.static_density = 1 if static else 0
        d.frozen = 0 if evolution else 1
        keep = []
        if piecewise_z is not None:
            z = np.ascontiguousarray(piecewise_z, dtype=np.float32)
            fz = np.ascontiguousarray(piecewise_fz, dtype=np.float32)
            assert z.shape == fz.shape
            keep += [z, fz]
            d.npiece = z.size
            d.piecewise_z = z.ctypes.data_as(C.POINTER(C.c_float))
            d.piecewise_fz = fz.ctypes.data_as(C.POINTER(C.c_float))
        d.seed = int(seed)
        for a in range(2):
            d.alpha[a], d.beta[a], d.emittance[a] = alpha[a], beta[a], emittance[a]
            d.range_x[a], d.range_y[a], d.range_z[a] = range_x[a], range_y[a], range_z[a]
        if file_name is not None:
            d.file_name = str(file_name).encode()
        d.n0, d.r1, d.r2 = n0, r1, r2
        h = C.c_void_p()
        ctx._check(ctx._L.qp_beam_create(ctx.h, C.byref(d), C.byref(h)))
        del keep
        self.ctx, self.h = ctx, h

    def np(self):
        return int(self.ctx._L.qp_beam_np(self.h))

    def qdp(self, q=None, slice=None):
        if q is None:
            self.ctx._check(self.ctx._L.qp_beam_qdp(self.h))
        else:
            self.ctx._check(self.ctx._L.qp_beam_qdpcopy(self.h, q.h, slice))

    def push(self, sim, dt):
        """beam3d%push with the 3D fields of `sim`'s last step (conducting boundaries)."""
        self.ctx._check(self.ctx._L.qp_beam_push(self.h, sim.h, C.c_float(dt)))

    def get_particles(self):
        out = np.zeros((7, self.np()), dtype=np.float32, order="F")
        self.ctx._check(self.ctx._L.qp_beam_download(self.h, _ptr(out)))
        return out

    def set_particles(self, part):
        """Upload part(7, np) (Fortran order, float32; pinned memory makes it async)."""
        assert part.dtype == np.float32 and part.flags["F_CONTIGUOUS"] and part.shape[0] == 7
        self.ctx._check(self.ctx._L.qp_beam_upload(self.h, _ptr(part),
                                                   C.c_longlong(part.shape[1])))

    def write_restart(self, dir, beam=1, rank=0, step=0):
        """beam3d%wrst: dir/RST/Beam-NNNN/RST-beamNNNN-RRRRRRRRRR_SSSSSSSS.qprst"""
        self.ctx._check(self.ctx._L.qp_beam_write_restart(self.h, dir.encode(), beam, rank, step))

    def read_restart(self, dir, beam=1, rank=0, step=0):
        """beam3d%rrst: replaces the particles with the restart file's."""
        self.ctx._check(self.ctx._L.qp_beam_read_restart(self.h, dir.encode(), beam, rank, step))

    def get_q3d(self):
        c = self.ctx
        out = np.zeros((c.nx + 2, c.ny + 1, c.nz + 1), dtype=np.float32, order="F")
        c._check(c._L.qp_beam_download_q3d(self.h, _ptr(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.ctx._L.qp_beam_destroy(self.h)
            self.h = None


class Simulation:
    """The fused 3D step: beam deposit, every slice, species renew, on the GPU."""

    def __init__(self, ctx: Context, species, beams, iter=2, store3d=True, use_graphs=False,
                 dt=0.0, tol=0.0, vpot=False, predict=False):
        d = _SimDesc()
        d.iter = iter  # passes per slice; with tol > 0 the most passes a slice may take
        d.tol = tol  # > 0: stop a slice's passes once |d epw| / |epw| <= tol
        d.vpot = 1 if vpot else 0  # keep the 3D vector potential ("vpot")
        # start B from 2 epw(j-1) - epw(j-2) (True or 1) or 3 epw(j-1) - 3 epw(j-2) + epw(j-3) (2)
        d.predict = int(predict)
        d.store3d = 1 if store3d else 0
        d.use_graphs = 1 if use_graphs else 0
        d.dt = dt  # 3D time step; > 0 ends every step with the beam push
        sp = (C.c_void_p * len(species))(*[s.h for s in species])
        bm = (C.c_void_p * max(len(beams), 1))(*[b.h for b in beams])
        h = C.c_void_p()
        ctx._check(ctx._L.qp_sim_create(ctx.h, C.byref(d), sp, len(species), bm, len(beams),
                                        C.byref(h)))
        self.ctx, self.h = ctx, h
        self.species, self.beams = species, beams

    def step3d(self) -> StepStats:
        st = StepStats()
        self.ctx._check(self.ctx._L.qp_sim_step3d(self.h, C.byref(st)))
        return st

    # the 3D step in the parts of go_simulation (simulation_class.f03:611-764)
    def begin3d(self):
        """Beam deposits, the fields handed to slice 1, slice cursor at 1."""
        self.ctx._check(self.ctx._L.qp_sim_begin3d(self.h))

    def slices(self, n=1):
        """Run the next n slices of the step."""
        self.ctx._check(self.ctx._L.qp_sim_slices(self.h, int(n)))

    def end3d(self) -> StepStats:
        """Beam push (dt > 0) and species renew, after all nz slices."""
        st = StepStats()
        self.ctx._check(self.ctx._L.qp_sim_end3d(self.h, C.byref(st)))
        return st

    @property
    def next_slice(self):
        """The slice the next slices() call starts with; 0 outside a step."""
        return int(self.ctx._L.qp_sim_next_slice(self.h))

    @property
    def graph_captures(self):
        """With use_graphs: the slice graphs captured so far."""
        return int(self.ctx._L.qp_sim_graph_captures(self.h))

    def set_field(self, name, arr):
        """Restore a field handed from slice to slice ("epw", "cu_k",
        "epw_prev", "epw_prev2"), reference k-space layout (dim, ny+1, nx+1)."""
        a = np.asfortranarray(arr, dtype=np.float32)
        self.ctx._check(self.ctx._L.qp_sim_upload_field(self.h, name.encode(), _ptr(a)))

    def get_plane(self, name, plane):
        """Plane `plane` (0..nz) of "bexyz", "bbxyz", "vpot" (3, nx+2, ny+1) or
        "q3", "qb" (nx+2, ny+1)."""
        c = self.ctx
        shape = (c.nx + 2, c.ny + 1) if name in ("q3", "qb") else (3, c.nx + 2, c.ny + 1)
        out = np.zeros(shape, dtype=np.float32, order="F")
        c._check(c._L.qp_sim_download_plane(self.h, name.encode(), int(plane), _ptr(out)))
        return out

    def get_field(self, name):
        c = self.ctx
        dims = dict(psi=1, fxy=2, bxyz=3, psit=1, cu=3, dcu=2, amu=3, epw=2, cu_k=3, epwb=2,
                    epw_prev=2, epw_prev2=2)
        dim = dims[name]
        ks = ("epw", "cu_k", "epwb", "epw_prev", "epw_prev2")
        shape = c.ks_shape(dim) if name in ks else c.rs_shape(dim)
        out = np.zeros(shape, dtype=np.float32, order="F")
        c._check(c._L.qp_sim_download_field(self.h, name.encode(), _ptr(out)))
        return out

    def get_3d(self, name):
        c = self.ctx
        if name == "q3":
            shape = (c.nx + 2, c.ny + 1, c.nz + 1)
        else:
            shape = (3, c.nx + 2, c.ny + 1, c.nz + 1)
        out = np.zeros(shape, dtype=np.float32, order="F")
        c._check(c._L.qp_sim_download_3d(self.h, name.encode(), _ptr(out)))
        return out

    def lineout(self, comp=3, out=None):
        """On-axis bexyz(comp) for every slice (nz+1 values)."""
        if out is None:
            out = np.zeros(self.ctx.nz + 1, dtype=np.float32)
        self.ctx._check(self.ctx._L.qp_sim_download_lineout(self.h, comp, _ptr(out)))
        return out

    def record(self, data):
        """Record one training pair per slice into `data` (a TrainingSet) from
        the next step on; None stops."""
        self.ctx._check(self.ctx._L.qp_sim_record(self.h, data.h if data is not None else None))
        self._rec = data

    def set_predictor(self, net):
        """The network that starts each slice's passes (predict=3)."""
        self.ctx._check(self.ctx._L.qp_sim_set_predictor(self.h, net.h))
        self._net = net

    def profile(self, nslices):
        """{kernel name: (total ms, launches, algorithmic bytes)} of nslices slices
        sampled across one whole 3D step (which it runs, advancing the
        simulation); launches of skipped passes are named "<kernel>:skipped"."""
        buf = C.create_string_buffer(4096)
        ms = (C.c_double * 64)()
        cnt = (C.c_int * 64)()
        byt = (C.c_double * 64)()
        n = self.ctx._check(self.ctx._L.qp_sim_profile(self.h, nslices, buf, 4096, ms, cnt, byt,
                                                       64))
        names = buf.value.decode().split("\n")[:n]
        return {names[i]: (ms[i], cnt[i], byt[i]) for i in range(n)}

    def close(self):
        if getattr(self, "h", None):
            self.ctx._L.qp_sim_destroy(self.h)
            self.h = None


class _ScanDesc(C.Structure):
    _fields_ = [("steps", C.c_int), ("workers", C.c_int)]


class ScanStats(C.Structure):
    _fields_ = [("gpu_ms", C.c_double), ("particle_slices", C.c_longlong),
                ("workers", C.c_int), ("failed", C.c_int)]


def _sim_array(sims):
    if not sims:
        raise QPError("scan: no instances")
    arr = (C.c_void_p * len(sims))(*[s.h for s in sims])
    return arr


def scan_run(sims, steps=1, workers=0) -> ScanStats:
    """Advance independent simulations (each on its own Context) by `steps` 3D
    steps; `workers` host threads step them concurrently on their own streams
    (0 = one per instance, 1 = one after another).  Device-timed."""
    L = lib()
    d = _ScanDesc(int(steps), int(workers))
    st = ScanStats()
    rc = L.qp_scan_run(_sim_array(sims), len(sims), C.byref(d), C.byref(st))
    if rc < 0:
        msg = L.qp_ctx_last_error(None)
        raise QPError(msg.decode() if msg else f"qpgpu error {rc}")
    return st


def scan_tune(sims, probe_steps=1):
    """The autotuner of the scan's concurrency: (best worker count, its
    particle-slices/s).  Advances every instance by probe_steps per candidate."""
    L = lib()
    w = C.c_int(0)
    r = C.c_double(0.0)
    rc = L.qp_scan_tune(_sim_array(sims), len(sims), int(probe_steps), C.byref(w), C.byref(r))
    if rc < 0:
        msg = L.qp_ctx_last_error(None)
        raise QPError(msg.decode() if msg else f"qpgpu error {rc}")
    return w.value, r.value


class _TrainDesc(C.Structure):
    _fields_ = [("steps", C.c_int), ("batch", C.c_int), ("lr", C.c_float),
                ("reserved", C.c_int), ("seed", C.c_ulonglong)]


class TrainStats(C.Structure):
    _fields_ = [("first_loss", C.c_double), ("last_loss", C.c_double), ("gpu_ms", C.c_double),
                ("steps", C.c_int), ("reserved", C.c_int)]


def _nn_check(rc):
    if rc < 0:
        msg = lib().qp_ctx_last_error(None)
        raise QPError(msg.decode() if msg else f"qpgpu error {rc}")
    return rc


class Predictor:
    """The learned start of the B passes: 5 layers of 3x3 convolutions (32
    channels, BF16 tensor cores) on Fourier-space images.  No counterpart in
    the reference, whose passes start from the previous slice's B
    (simulation_class.f03:676)."""

    def __init__(self, device=0, seed=1):
        h = C.c_void_p()
        _nn_check(lib().qp_nn_create(device, C.c_ulonglong(seed), C.byref(h)))
        self.h = h

    @property
    def nparams(self):
        return int(lib().qp_nn_num_params(self.h))

    def get_params(self):
        out = np.zeros(self.nparams, dtype=np.float32)
        _nn_check(lib().qp_nn_get_params(self.h, _ptr(out)))
        return out

    def set_params(self, p):
        a = np.ascontiguousarray(p, dtype=np.float32)
        assert a.size == self.nparams
        _nn_check(lib().qp_nn_set_params(self.h, _ptr(a)))

    def forward(self, x):
        """x[nb][16][h][w] (w a multiple of 128) -> out[nb][2][h][w]."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        nb, _, hh, ww = x.shape
        out = np.zeros((nb, 2, hh, ww), dtype=np.float32)
        _nn_check(lib().qp_nn_forward(self.h, _ptr(x), nb, hh, ww, _ptr(out)))
        return out

    def loss_grad(self, x, target):
        """(mean squared error, gradient of every parameter)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(target, dtype=np.float32)
        nb, _, hh, ww = x.shape
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = C.c_double(0.0)
        _nn_check(lib().qp_nn_loss_grad(self.h, _ptr(x), _ptr(t), nb, hh, ww, C.byref(loss),
                                        _ptr(g)))
        return loss.value, g

    def train(self, data, steps=500, batch=16, lr=1e-3, seed=7) -> TrainStats:
        d = _TrainDesc(int(steps), int(batch), float(lr), 0, int(seed))
        st = TrainStats()
        _nn_check(lib().qp_nn_train(self.h, data.h, C.byref(d), C.byref(st)))
        return st

    def close(self):
        if getattr(self, "h", None):
            lib().qp_nn_destroy(self.h)
            self.h = None


class TrainingSet:
    """Training pairs recorded from simulations (Simulation.record)."""

    def __init__(self, capacity, device=0):
        h = C.c_void_p()
        _nn_check(lib().qp_nn_data_create(device, int(capacity), C.byref(h)))
        self.h = h
        self.capacity = int(capacity)

    def __len__(self):
        return int(lib().qp_nn_data_count(self.h))

    def get(self, i):
        """(features [16][128][128], target [2][128][128], scale) of pair i."""
        img = np.zeros((16, 128, 128), dtype=np.float32)
        tgt = np.zeros((2, 128, 128), dtype=np.float32)
        sc = np.zeros(1, dtype=np.float32)
        _nn_check(lib().qp_nn_data_get(self.h, int(i), _ptr(img), _ptr(tgt), _ptr(sc)))
        return img, tgt, float(sc[0])

    def close(self):
        if getattr(self, "h", None):
            lib().qp_nn_data_destroy(self.h)
            self.h = None
