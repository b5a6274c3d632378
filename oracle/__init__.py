"""CPU oracle for the qqcd solver hot path -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper of oracle/_build/liboracle.so, the line-by-line C++ restatement of the
reference Fortran routines (see oracle/oracle.h for the file:line of each).  Parity is
UNPINNED against the Fortran itself (no Fortran compiler here, and the reference ships
no golden vectors); it is pinned against analytic known answers and scipy LAPACK in
tests/.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
LIB_OMP = HERE / "_build" / "liboracle_omp.so"  # timing build (OpenMP site loops)

_lib = None
_use = LIB


def build() -> Path:
    srcs = list(HERE.glob("*.cpp")) + list(HERE.glob("*.h")) + [HERE / "Makefile"]
    newest = max(p.stat().st_mtime for p in srcs)
    if any(not f.exists() or f.stat().st_mtime < newest for f in (LIB, LIB_OMP)):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def use_timing_build(threads: int | None = None) -> int:
    """Load the OpenMP timing build (CPU-baseline legs of bench.py only; the parity
    tests use the serial build).  Must come before the first oracle call of the
    process.  Returns the number of host threads it will use."""
    global _use
    if _lib is not None and _use != LIB_OMP:
        raise RuntimeError("the serial oracle is already loaded in this process")
    _use = LIB_OMP
    L = lib()
    if threads:
        L.oq_set_threads(int(threads))
    return int(L.oq_threads())


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(_use))
        P, I, D = C.c_void_p, C.c_int, C.c_double
        IP, DP = C.POINTER(C.c_int), C.POINTER(C.c_double)
        sig = {
            "oq_geom_create": ([I, I, I, I, IP, DP, DP], P),
            "oq_geom_destroy": ([P], None),
            "oq_nvhalf": ([P], I), "oq_ntotal": ([P], I), "oq_nbmax": ([P], I),
            "oq_tables": ([P, IP, IP, IP, IP, IP, IP, IP, IP], None),
            "oq_set_coact": ([P, DP, DP], None),
            "oq_site_of_coords": ([P, IP, IP, IP, IP, IP, IP], None),
            "oq_initlagfib": ([I, I], None),
            "oq_rnds": ([I, DP], None),
            "oq_lagfib_state": ([IP, IP, IP], None),
            "oq_lagfib_set_state": ([IP, I, I], None),
            "oq_pointsource": ([P, DP, DP, IP, I, I], None),
            "oq_z2source": ([P, DP, DP], None),
            "oq_z4source": ([P, DP, DP], None),
            "oq_hsingle": ([P, DP, DP, DP, I, I], None),
            "oq_hdouble": ([P, DP, DP, DP, I, D], None),
            "oq_hdbletm": ([P, DP, DP, DP, I, DP], None),
            "oq_twmshift": ([P, DP, DP, DP, I, DP], None),
            "oq_gamma5mult": ([P, DP, DP, DP, I, DP], None),
            "oq_gam5x": ([P, DP], None),
            "oq_gamma5vector": ([P, DP, I], None),
            "oq_vecdot": ([P, DP, DP, DP], None),
            "oq_defl_create": ([P, I, I], P),
            "oq_defl_destroy": ([P], None),
            "oq_defl_get": ([P, I, DP, DP], None),
            "oq_gmresdr": ([P, DP, DP, IP, D, I, DP, DP, P, P], I),
            "oq_gmresdrshift": ([P, DP, DP, I, DP, IP, D, I, DP, DP, DP, P], I),
            "oq_gmresproject": ([P, DP, DP, IP, D, I, DP, DP, I, P, P], I),
            "oq_psc": ([P, DP, DP, IP, D, I, DP, DP, I, P, P], I),
            "oq_bicgstab": ([P, DP, DP, D, I, DP, DP, P, I], I),
            "oq_fermprop": ([P, DP, DP, DP, I, D, I, IP, DP, DP, DP, I, I, P, P], I),
            "oq_linearsolver": ([I, I, DP, I, IP, DP, I], None),
            "oq_hessenberg": ([DP, I, I, I, I, DP], None),
            "oq_qgenerator": ([I, I, I, DP, I, DP], None),
            "oq_evalues": ([I, I, I, I, DP, I, DP, DP, I], None),
            "oq_orgschur": ([IP, I, DP, I, DP, I, DP, IP], None),
            "oq_twaverage_level0": ([P, DP, DP, DP, DP, DP, D, D, C.c_int, DP], None),
            "oq_twvev": ([P, DP, D, D, IP, I, I, I, I, I, DP], None),
            "oq_vevw": ([P, DP, IP, D, DP, DP, DP], I),
            "oq_average": ([P, DP, DP, DP, DP, DP, D, I, I, I, DP, DP], None),
            "oq_momfacs": ([P, IP, DP], None),
            "oq_eigmodes": ([P, DP, I, IP, I, DP, DP, DP, DP, DP, DP, IP], I),
            "oq_xigenerator": ([P, DP, I, D, DP, DP, I, DP], None),
            "oq_eigaverage": ([P, DP, I, I, I, DP, DP, D, DP, DP, DP, I, DP], None),
            "oq_loop_slices": ([P, DP, DP, DP, DP, DP, I, D, DP], None),
            "oq_smear": ([P, DP, DP, DP, DP, DP, D, I], None),
            "oq_mesoncorr": ([P, DP, DP, IP, I, DP, DP], None),
            "oq_ppcoeffs": ([P, DP, DP, DP, D, I, DP], None),
            "oq_ppaverage": ([P, DP, I, DP, DP, DP, DP, DP, D, I, DP], None),
            "oq_xipolygenerator": ([P, DP, I, D, DP, DP, DP, DP], None),
            "oq_generalaverage": ([P, DP, I, DP, DP, DP, I, DP, DP, DP, DP, DP, DP, D, I, I, DP, DP, DP, DP,
                                   DP], None),
            "oq_twaverage_mom": ([P, DP, DP, DP, DP, DP, D, D, IP, I, I, I, DP], None),
            "oq_twvev_sites": ([P, DP, D, D, IP, I, I, I, IP, I, DP], None),
            "oq_set_kcyclim": ([I], None),
            "oq_set_threads": ([I], None),
            "oq_threads": ([], I),
            "oq_coldstart": ([P, DP], None),
            "oq_heatbath": ([P, DP, D, I, I, DP], None),
            "oq_aveplaq": ([P, DP], D),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int))


class SolveLog(C.Structure):
    _fields_ = [("itercount", C.c_int), ("mvp", C.c_int), ("ncycles", C.c_int), ("nhist", C.c_int),
                ("hist", C.c_double * 4096), ("hist_mvp", C.c_int * 4096), ("nritz", C.c_int),
                ("ritz", C.c_double * 1024), ("final_rel", C.c_double)]

    def history(self):
        n = self.nhist
        return np.array(self.hist[:n]), np.array(self.hist_mvp[:n])

    def ritz_values(self):
        r = np.array(self.ritz[: 2 * self.nritz]).reshape(-1, 2)
        return r[:, 0] + 1j * r[:, 1]


class OracleLattice:
    """The reference's single-process lattice (nps = 1) with index tables and gauge field."""

    def __init__(self, nx, ny, nz, nt, bc=(1, 1, 1, -1), c1=(1.0,) * 4, c2=(1.0,) * 4):
        L = lib()
        self._bc = np.array(bc, np.int32)
        self._c1 = np.array(c1, np.float64)
        self._c2 = np.array(c2, np.float64)
        self._g = L.oq_geom_create(nx, ny, nz, nt, self._bc.ctypes.data_as(C.POINTER(C.c_int)),
                                   _dp(self._c1), _dp(self._c2))
        if not self._g:
            raise ValueError("lattice extents must be multiples of 4")
        self.dims = (nx, ny, nz, nt)
        self.nvhalf = L.oq_nvhalf(self._g)
        self.ntotal = L.oq_ntotal(self._g)
        self.u = None

    def __del__(self):
        try:
            if self._g:
                lib().oq_geom_destroy(self._g)
        except Exception:
            pass

    @property
    def half_shape(self):
        return (8, 2, 4, self.ntotal, 6)

    @property
    def gauge_shape(self):
        return (16, 2, 4, self.ntotal, 18)

    def new_half(self):
        return np.zeros(self.half_shape)

    def set_gauge(self, u: np.ndarray):
        assert u.shape == self.gauge_shape
        self.u = np.ascontiguousarray(u, dtype=np.float64)

    def set_coact(self, c1, c2):
        self._c1 = np.array(c1, np.float64)
        self._c2 = np.array(c2, np.float64)
        lib().oq_set_coact(self._g, _dp(self._c1), _dp(self._c2))

    def site_of_coords(self, x):
        x, xp = _ip(x)
        out = [C.c_int() for _ in range(5)]
        lib().oq_site_of_coords(self._g, xp, *[C.byref(o) for o in out])
        return tuple(o.value for o in out)  # isite, ieo, ibl, gblclr, ibleo

    # ---- Dirac operator ----
    def hsingle(self, gin, idag, gblclr):
        out = self.new_half()
        gi = np.array(gin, dtype=np.float64, copy=True)
        lib().oq_hsingle(self._g, _dp(out), _dp(self.u), _dp(gi), idag, gblclr)
        return out

    def hdouble(self, ge, idag, kappa):
        out = self.new_half()
        gi = np.array(ge, dtype=np.float64, copy=True)
        lib().oq_hdouble(self._g, _dp(out), _dp(self.u), _dp(gi), idag, float(kappa))
        return out

    def hdbletm(self, ge, idag, kappa):
        out = self.new_half()
        gi = np.array(ge, dtype=np.float64, copy=True)
        k = np.array(kappa, np.float64)
        lib().oq_hdbletm(self._g, _dp(out), _dp(self.u), _dp(gi), idag, _dp(k))
        return out

    def twmshift(self, gwhole, idag, kappa):
        out = np.zeros((2,) + self.half_shape)
        gi = np.array(gwhole, dtype=np.float64, copy=True)
        k = np.array(kappa, np.float64)
        lib().oq_twmshift(self._g, _dp(out), _dp(self.u), _dp(gi), idag, _dp(k))
        return out

    def gamma5mult(self, ge, idag, kappa):
        out = self.new_half()
        gi = np.array(ge, dtype=np.float64, copy=True)
        k = np.array(kappa, np.float64)
        lib().oq_gamma5mult(self._g, _dp(out), _dp(self.u), _dp(gi), idag, _dp(k))
        return out

    def vecdot(self, a, b):
        r = np.zeros(2)
        lib().oq_vecdot(self._g, _dp(np.ascontiguousarray(a)), _dp(np.ascontiguousarray(b)), _dp(r))
        return complex(r[0], r[1])

    def gam5x(self, a):
        a = np.array(a, dtype=np.float64, copy=True)
        lib().oq_gam5x(self._g, _dp(a))
        return a

    # ---- inverters ----
    def deflation(self, nmax, kmax):
        return lib().oq_defl_create(self._g, nmax, kmax)

    def defl_get(self, d, k, nmax):
        vt = np.zeros((k + 1,) + self.half_shape)
        hc = np.zeros((k, k + 1, 2))
        lib().oq_defl_get(d, k, _dp(vt), _dp(hc))
        return vt, hc[..., 0] .T + 1j * hc[..., 1].T

    def gmresdr(self, phi, x, GMRES, resmax, itermin=0, kappa=(0.15, 0.0), defl=None):
        x = np.array(x, dtype=np.float64, copy=True)
        log = SolveLog()
        G, Gp = _ip(GMRES)
        k = np.array(kappa, np.float64)
        st = lib().oq_gmresdr(self._g, _dp(np.ascontiguousarray(phi)), _dp(x), Gp, float(resmax), itermin,
                              _dp(self.u), _dp(k), defl, C.byref(log))
        return x, st, log

    def gmresdrshift(self, b, sigma, GMRES, resmax, itermin=0, kappa=(0.15, 0.01)):
        """Solutions of (A - sigma_s) x_s = b, A = gamma5mult; returns (x[ns], status,
        resid[ns] (absolute, recursively updated), log)."""
        sig = np.ascontiguousarray(sigma, dtype=np.float64)
        ns = len(sig)
        x = np.zeros((ns,) + self.half_shape)
        resid = np.zeros(ns)
        log = SolveLog()
        G, Gp = _ip(GMRES)
        k = np.array(kappa, np.float64)
        st = lib().oq_gmresdrshift(self._g, _dp(np.ascontiguousarray(b)), _dp(x), ns, _dp(sig), Gp,
                                   float(resmax), itermin, _dp(self.u), _dp(k), _dp(resid), C.byref(log))
        return x, st, resid, log

    def gmresproject(self, b, GMRES, resmax, itermin=0, kappa=(0.15, 0.0), isignal=2, defl=None):
        x = self.new_half()
        log = SolveLog()
        G, Gp = _ip(GMRES)
        k = np.array(kappa, np.float64)
        st = lib().oq_gmresproject(self._g, _dp(np.ascontiguousarray(b)), _dp(x), Gp, float(resmax), itermin,
                                   _dp(self.u), _dp(k), isignal, defl, C.byref(log))
        return x, st, log

    def psc(self, b, x, GMRES, resmax, itermin=0, kappa=(0.15, 0.0), isignal=1, defl=None):
        x = np.array(x, dtype=np.float64, copy=True)
        log = SolveLog()
        G, Gp = _ip(GMRES)
        k = np.array(kappa, np.float64)
        st = lib().oq_psc(self._g, _dp(np.ascontiguousarray(b)), _dp(x), Gp, float(resmax), itermin,
                          _dp(self.u), _dp(k), isignal, defl, C.byref(log))
        return x, st, log

    def bicgstab(self, phi, x, resmax, itermin=0, kappa=(0.15, 0.0), maxiter=0):
        x = np.array(x, dtype=np.float64, copy=True)
        log = SolveLog()
        k = np.array(kappa, np.float64)
        st = lib().oq_bicgstab(self._g, _dp(np.ascontiguousarray(phi)), _dp(x), float(resmax), itermin,
                               _dp(self.u), _dp(k), C.byref(log), maxiter)
        return x, st, log

    def fermprop(self, be, bo, kappa, inverter=5, resmax=1e-10, itermin=0, nGMRES=(30, 10), ntmqcd=0,
                 isignal=1, defl=None, xe=None):
        xe = self.new_half() if xe is None else np.array(xe, dtype=np.float64, copy=True)
        xo = self.new_half()
        bo = np.array(bo, dtype=np.float64, copy=True)
        log = SolveLog()
        G, Gp = _ip(nGMRES)
        k = np.array(kappa, np.float64)
        st = lib().oq_fermprop(self._g, _dp(np.ascontiguousarray(be)), _dp(bo), _dp(k), inverter, float(resmax),
                               itermin, Gp, _dp(self.u), _dp(xe), _dp(xo), ntmqcd, isignal, defl,
                               C.byref(log))
        return xe, xo, st, log

    # ---- sources ----
    def pointsource(self, src, icsrc, idsrc):
        be, bo = self.new_half(), self.new_half()
        s, sp = _ip(src)
        lib().oq_pointsource(self._g, _dp(be), _dp(bo), sp, icsrc, idsrc)
        return be, bo

    def z2source(self):
        be, bo = self.new_half(), self.new_half()
        lib().oq_z2source(self._g, _dp(be), _dp(bo))
        return be, bo

    def z4source(self):
        be, bo = self.new_half(), self.new_half()
        lib().oq_z4source(self._g, _dp(be), _dp(bo))
        return be, bo

    def twaverage_level0(self, be, bo, xe, xo, kappa, delta=0.0, dobndry=0):
        """Level-0 traces of one noise: J[iop, t, re/im] (twAverage, nsub = 0)."""
        J = np.zeros((6, self.dims[3], 2))
        lib().oq_twaverage_level0(self._g, _dp(np.ascontiguousarray(be)), _dp(np.ascontiguousarray(bo)),
                                  _dp(np.ascontiguousarray(xe)), _dp(np.ascontiguousarray(xo)),
                                  _dp(self.u), float(kappa), float(delta), int(dobndry), _dp(J))
        return J

    def twaverage(self, be, bo, xe, xo, kappa, delta=0.0, io=(1, 1, 1), dobndry=0, nmom=5, ir=1):
        """Level-0 traces of one noise with twAverage's momentum projections:
        J[iop, imom, t, re/im] (the reverse of (2, nt, nmom, 6)), ops other than 2 and
        6 scaled by kappa."""
        J = np.zeros((6, nmom, self.dims[3], 2))
        _, iop = _ip(io)
        lib().oq_twaverage_mom(self._g, _dp(np.ascontiguousarray(be)), _dp(np.ascontiguousarray(bo)),
                               _dp(np.ascontiguousarray(xe)), _dp(np.ascontiguousarray(xo)), _dp(self.u),
                               float(kappa), float(delta), iop, int(dobndry), int(nmom), int(ir), _dp(J))
        return J

    def momfacs(self, io=(1, 1, 1)):
        """momfacs (Q/disconloops.f90:8925-8984): numpy shape (5, 4, 16, 2, nvhalf)."""
        mf = np.zeros((5, 4, 16, 2, self.nvhalf))
        _, iop = _ip(io)
        lib().oq_momfacs(self._g, iop, _dp(mf))
        return mf

    def average(self, be, bo, xe, xo, kappa, nsub=6, nmom=5, nop=9, momfac=None):
        """average (Q/disconloops.f90:5343-5733): the Wilson loop operators of one noise at
        subtraction levels 1..nsub.  momfac has the reference's shape (nvhalf, 2, 16,
        nmom-1, >= 5) in Fortran order, i.e. numpy shape (>= 5, nmom-1, 16, 2, nvhalf).
        Returns Jtime as (nop, nmom, nsub, nt, 2)."""
        J = np.zeros((nop, nmom, nsub, self.dims[3], 2))
        mf = np.zeros(1) if momfac is None else np.ascontiguousarray(momfac, dtype=np.float64)
        lib().oq_average(self._g, _dp(self.u), _dp(np.ascontiguousarray(be)), _dp(np.ascontiguousarray(bo)),
                         _dp(np.ascontiguousarray(xe)), _dp(np.ascontiguousarray(xo)), float(kappa), int(nsub),
                         int(nmom), int(nop), _dp(mf), _dp(J))
        return J

    def eigmodes(self, kind, nGMRES, ncycles, kappa, se=None, so=None):
        """eigmodesofM (kind 1) / eigmodesofMprime (kind 2), Q/disconloops.f90:1593-1937,
        2573-2875.  Returns (evals complex (numEV,), R, L) with R, L of numpy shape
        (numEV, 2) + half_shape (even then odd half), and the cycles run."""
        k = int(nGMRES[1])
        R = np.zeros((k, 2) + self.half_shape)
        L = np.zeros((k, 2) + self.half_shape)
        ev = np.zeros(2 * k)
        cyc = C.c_int(0)
        _, gp = _ip(nGMRES)
        kp = np.ascontiguousarray(kappa, dtype=np.float64)
        z = np.zeros(self.half_shape)
        se = z if se is None else np.ascontiguousarray(se)
        so = z if so is None else np.ascontiguousarray(so)
        n = lib().oq_eigmodes(self._g, _dp(self.u), int(kind), gp, int(ncycles), _dp(kp), _dp(se), _dp(so),
                              _dp(R), _dp(L), _dp(ev), C.byref(cyc))
        return ev[0:2 * n:2] + 1j * ev[1:2 * n:2], R[:n].copy(), L[:n].copy(), cyc.value

    def xigenerator(self, R, L, kappa, gammaid):
        """xigenerator (Q/disconloops.f90:465-838): xiinv as complex (numEV, 6)."""
        n = R.shape[0]
        xi = np.zeros((n, 6, 2))
        lib().oq_xigenerator(self._g, _dp(self.u), n, float(kappa), _dp(np.ascontiguousarray(R)),
                             _dp(np.ascontiguousarray(L)), int(gammaid), _dp(xi))
        return xi[..., 0] + 1j * xi[..., 1]

    def eigaverage(self, ze, zo, kappa, R, L, scal, eshfes, eigstart=1, eigstep=1):
        """eigaverage (Q/disconloops.f90:3239-3342) at imom = 1: Jtime as (9, numEV, nt, 2)."""
        n = R.shape[0]
        J = np.zeros((9, n, self.dims[3], 2))
        s = np.zeros((n, 2))
        s[:, 0] = np.real(scal)
        s[:, 1] = np.imag(scal)
        lib().oq_eigaverage(self._g, _dp(self.u), n, int(eigstart), int(eigstep), _dp(np.ascontiguousarray(ze)),
                            _dp(np.ascontiguousarray(zo)), float(kappa), _dp(np.ascontiguousarray(R)),
                            _dp(np.ascontiguousarray(L)), _dp(s), int(eshfes), _dp(J))
        return J

    def ppcoeffs(self, be, bo, kappa, p):
        """The least-squares polynomial of ppaverage* (complex (p,))."""
        co = np.zeros((p, 2))
        lib().oq_ppcoeffs(self._g, _dp(self.u), _dp(np.ascontiguousarray(be)), _dp(np.ascontiguousarray(bo)),
                          float(kappa), int(p), _dp(co))
        return co[:, 0] + 1j * co[:, 1]

    @staticmethod
    def _cplx2(a):
        a = np.asarray(a, complex)
        out = np.zeros((len(a), 2))
        out[:, 0], out[:, 1] = a.real, a.imag
        return out

    def ppaverage(self, p, co, be, bo, xe, xo, kappa, nsub=6):
        """ppaverage (p = 5) / ppaverage1 (8) / ppaverage2 (11) at imom = 1: (9, nsub, nt, 2)."""
        J = np.zeros((9, nsub, self.dims[3], 2))
        lib().oq_ppaverage(self._g, _dp(self.u), int(p), _dp(self._cplx2(co)), _dp(np.ascontiguousarray(be)),
                           _dp(np.ascontiguousarray(bo)), _dp(np.ascontiguousarray(xe)),
                           _dp(np.ascontiguousarray(xo)), float(kappa), int(nsub), _dp(J))
        return J

    def xipolygenerator(self, R, L, kappa, co):
        n = R.shape[0]
        xi = np.zeros((n, 6, 2))
        lib().oq_xipolygenerator(self._g, _dp(self.u), n, float(kappa), _dp(np.ascontiguousarray(R)),
                                 _dp(np.ascontiguousarray(L)), _dp(self._cplx2(co)), _dp(xi))
        return xi[..., 0] + 1j * xi[..., 1]

    def loop_slices(self, be, bo, ye, yo, ksub, kappa):
        J = np.zeros((9, self.dims[3], 2))
        lib().oq_loop_slices(self._g, _dp(self.u), _dp(np.ascontiguousarray(be)), _dp(np.ascontiguousarray(bo)),
                             _dp(np.ascontiguousarray(ye)), _dp(np.ascontiguousarray(yo)), int(ksub), float(kappa),
                             _dp(J))
        return J

    def generalaverage(self, m, mp, ze, zo, xe, xo, kappa, co11, co8, co5, copoly, eigstart=1, eigstep=1):
        """generalaverage at imom = 1; m = (evals, R, L) of M, mp = (evals, R) of M gamma5.
        Returns Jave as (9, 10, numEV_MAX, 6, nt, 2)."""
        ev1, R1, L1 = m
        ev2, R2 = mp[0], mp[1]
        n1, n2 = len(ev1), len(ev2)
        ne = max(1, n1, n2)
        J = np.zeros((9, 10, ne, 6, self.dims[3], 2))
        z = np.zeros((1, 2) + self.half_shape)
        R1 = np.ascontiguousarray(R1 if n1 else z)
        L1 = np.ascontiguousarray(L1 if n1 else z)
        R2 = np.ascontiguousarray(R2 if n2 else z)
        lib().oq_generalaverage(self._g, _dp(self.u), n1, _dp(R1), _dp(L1), _dp(self._cplx2(ev1) if n1 else np.zeros((1, 2))),
                                n2, _dp(R2), _dp(self._cplx2(ev2) if n2 else np.zeros((1, 2))),
                                _dp(np.ascontiguousarray(ze)), _dp(np.ascontiguousarray(zo)),
                                _dp(np.ascontiguousarray(xe)), _dp(np.ascontiguousarray(xo)), float(kappa),
                                int(eigstart), int(eigstep), _dp(self._cplx2(co11)), _dp(self._cplx2(co8)),
                                _dp(self._cplx2(co5)), _dp(self._cplx2(copoly)), _dp(J))
        return J

    def smear(self, ge, go, asmear, nsmear):
        he, ho = self.new_half(), self.new_half()
        lib().oq_smear(self._g, _dp(self.u), _dp(he), _dp(ho), _dp(np.ascontiguousarray(ge)),
                       _dp(np.ascontiguousarray(go)), float(asmear), int(nsmear))
        return he, ho

    def mesoncorr(self, q, src, qbar=None, channels=0):
        """mesoncorr's correlators: q (12, 2) + half_shape; returns corrRe, corrIm as
        (28, 9, 9, 9, nt) numpy arrays (the reverse of the Fortran order)."""
        re = np.zeros((28, 9, 9, 9, self.dims[3]))
        im = np.zeros_like(re)
        _, sp = _ip(src)
        qb = np.ascontiguousarray(q if qbar is None else qbar)
        lib().oq_mesoncorr(self._g, _dp(np.ascontiguousarray(q)), _dp(qb), sp, int(channels), _dp(re), _dp(im))
        return re, im

    def twvev(self, kappa, delta=0.0, io=(1, 1, 1), dobndry=0, ir=1, nsub=6, nmom=5, nop=6):
        """twvev (Q/vevbleft.f90:757-2536) on the stored gauge field: Jvev as a numpy
        array of shape (nop, nmom, 6, nt, 2), the reverse of the Fortran (2, nt, 6, nmom,
        nop)."""
        J = np.zeros((nop, nmom, 6, self.dims[3], 2))
        _, iop = _ip(io)
        lib().oq_twvev(self._g, _dp(self.u), float(kappa), float(delta), iop, int(dobndry), int(ir), int(nsub),
                       int(nmom), int(nop), _dp(J))
        return J

    def vev(self, kappa, io=(1, 1, 1)):
        """vev (Q/disconloops.f90:4653-5339) on the stored gauge field: (Jvev, plaq, psi),
        Jvev as a numpy array of shape (5 op, 5 momenta, nt, 2), the reverse of the
        Fortran (2, nt, 5, 5)."""
        J = np.zeros((5, 5, self.dims[3], 2))
        plaq = np.zeros(1)
        psi = np.zeros(1)
        _, iop = _ip(io)
        rc = lib().oq_vevw(self._g, _dp(self.u), iop, float(kappa), _dp(J), _dp(plaq), _dp(psi))
        if rc != 0:
            raise RuntimeError("oq_vevw: site enumeration disagrees with the site map")
        return J, float(plaq[0]), float(psi[0])

    def twvev_sites(self, sites, kappa, delta=0.0, io=(1, 1, 1), dobndry=0, ir=1, nsub=6):
        """opertemp contributions of the listed 1-based lexicographic sites:
        array (isb 2, momentum 5, nt, op 12)."""
        O = np.zeros((2, 5, self.dims[3], 12))
        s, sp = _ip(sites)
        _, iop = _ip(io)
        lib().oq_twvev_sites(self._g, _dp(self.u), float(kappa), float(delta), iop, int(dobndry), int(ir),
                             int(nsub), sp, len(s), _dp(O))
        return O

    def pionrho(self, xe, xo, idsrc):
        """pionrho (Q/quark.f90:1033-1212), restated loop by loop for one process
        (npt = 1): the local pion, rho and decay correlators of one propagator column.
        Time slice it - 1 (ibleo 1..4) and it (ibleo 5..8) of the isite range of itbit
        (nsite = 2 nvhalf / nt sites per pair of slices); spins 1..4 with the signs of
        the reference's rbit and dbit; the gamma_5 spin rotation the reference applies
        at two slices leaves the sums of squares unchanged.  Returns (pion, rho, decay)."""
        nt = self.dims[3]
        nsite = 2 * self.nvhalf // nt
        pbit, rbit, dbit = np.zeros(nt), np.zeros(nt), np.zeros(nt)
        rs = np.array([1.0, -1.0, -1.0, 1.0])
        ds = np.array([1.0, 1.0, -1.0, -1.0])
        sitemin = 0
        for itbit in range(2, nt + 1, 2):
            it = itbit
            sl = slice(sitemin, sitemin + nsite)
            for ibleo in range(4):
                for ieo in range(2):
                    for half, tslot in ((ibleo, it - 2), (ibleo + 4, it - 1)):
                        sq = np.zeros(4)
                        for x in (xe, xo):
                            sq += np.sum(x[half, ieo, :, sl, :] ** 2, axis=(1, 2))
                        pbit[tslot] += sq.sum()
                        rbit[tslot] += np.dot(rs, sq)
                        dbit[tslot] += np.dot(ds, sq)
            sitemin += nsite
        rsgn = [1.0, -1.0, -1.0, 1.0][idsrc - 1]
        return pbit, rsgn * rbit, dbit

    # ---- gauge helpers ----
    def coldstart(self):
        u = np.zeros(self.gauge_shape)
        lib().oq_coldstart(self._g, _dp(u))
        return u

    def heatbath(self, u, beta, nsweeps, nhit=1):
        """The reference's pseudo-heatbath on u (reference layout, updated in place),
        drawing from the lagfib stream (call initlagfib first).  Returns the average
        plaquette after each sweep."""
        plaq = np.zeros(nsweeps)
        lib().oq_heatbath(self._g, _dp(u), float(beta), int(nsweeps), int(nhit), _dp(plaq))
        return plaq

    def aveplaq(self, u=None):
        u = self.u if u is None else u
        return lib().oq_aveplaq(self._g, _dp(np.ascontiguousarray(u)))


def set_kcyclim(n: int):
    """Cap GMRES-DR / GMRES-Proj cycles (0 restores the reference's 5000)."""
    lib().oq_set_kcyclim(int(n))


def initlagfib(myid: int, iseed: int):
    # bigdelay indexes c(ndelay) (G/lagfib.f90:185): a negative delay overruns it
    if not 0 <= myid + iseed < 2**31:
        raise ValueError("myid + iseed must be in [0, 2^31)")
    lib().oq_initlagfib(myid, iseed)


def rnds(m: int) -> np.ndarray:
    out = np.zeros(m)
    lib().oq_rnds(m, _dp(out))
    return out


# ---- restated pseudolapack, on complex numpy matrices ----
def _to_f(a: np.ndarray, ld: int | None = None) -> np.ndarray:
    m, n = a.shape
    ld = ld or m
    buf = np.zeros((n, ld, 2))
    buf[:, :m, 0] = a.real.T
    buf[:, :m, 1] = a.imag.T
    return buf


def _from_f(buf: np.ndarray, m: int) -> np.ndarray:
    return (buf[:, :m, 0] + 1j * buf[:, :m, 1]).T


def linearsolver(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    n = a.shape[0]
    A = _to_f(a)
    B = _to_f(b.reshape(n, -1))
    piv = np.zeros(n, np.int32)
    lib().oq_linearsolver(n, B.shape[0], _dp(A), n, piv.ctypes.data_as(C.POINTER(C.c_int)), _dp(B), n)
    return _from_f(B, n)


def schur_selected(h: np.ndarray, k: int):
    """gmresdr's harmonic-Ritz Schur step: hessenberg -> qgenerator -> evalues ->
    select the k smallest |theta| -> orgschur.  Returns (T, Z, w)."""
    n = h.shape[0]
    A = _to_f(h)
    tau = np.zeros((n, 2))
    lib().oq_hessenberg(_dp(A), n, n, 1, n, _dp(tau))
    Z = np.zeros_like(A)
    for j in range(n):
        Z[j, j:n] = A[j, j:n]
    lib().oq_qgenerator(n, 1, n, _dp(Z), n, _dp(tau))
    w = np.zeros((n, 2))
    lib().oq_evalues(1, n, 1, n, _dp(A), n, _dp(w), _dp(Z), n)
    wc = w[:, 0] + 1j * w[:, 1]
    mag = np.sort(np.abs(wc))
    sel = (np.abs(wc) <= mag[k - 1]).astype(np.int32)
    m = C.c_int()
    lib().oq_orgschur(sel.ctypes.data_as(C.POINTER(C.c_int)), n, _dp(A), n, _dp(Z), n, _dp(w), C.byref(m))
    return _from_f(A, n), _from_f(Z, n), w[:, 0] + 1j * w[:, 1], wc
