"""B200-native solver hot path of the BaylorLQCD ``qqcd`` code.

Python mirror of the reference's Fortran interface for the path (modules diracops,
inverters, quark and disconloops) over the C ABI of ``libqqcd_gpu.so``
(``include/qqcd_gpu.h``).  Arrays use the reference's own layouts:

* Dirac half-vector ``g(6, ntotal, 4, 2, 8)`` -> numpy shape ``(8, 2, 4, ntotal, 6)``
  (C order equals the Fortran column-major order);
* gauge field ``u(18, ntotal, 4, 2, 16)`` -> numpy shape ``(16, 2, 4, ntotal, 18)``.

Arrays may be numpy arrays (host) or torch CUDA tensors (device, zero copy).  There is
no CPU fallback: constructing a :class:`Lattice` without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libqqcd_gpu.so"

QQ_OK, QQ_NOT_CONVERGED, QQ_NAN, QQ_BAD_ARG, QQ_CUDA_ERR, QQ_ABORTED, QQ_NO_DEVICE, QQ_SINGULAR = range(8)
STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "NAN", 3: "BAD_ARG", 4: "CUDA_ERR", 5: "ABORTED",
                6: "NO_DEVICE", 7: "SINGULAR"}

# Every symbol of include/qqcd_gpu.h
EXPORTED = [
    "qq_ctx_create", "qq_ctx_destroy", "qq_ctx_dims", "qq_last_error", "qq_set_coact",
    "qq_gauge_upload", "qq_hsingle", "qq_hdouble", "qq_hdbletm", "qq_twmshift", "qq_gamma5mult", "qq_vecdot",
    "qq_vecdot_noalloc",
    "qq_defl_create", "qq_defl_destroy", "qq_defl_size", "qq_defl_vector", "qq_net_train_pairs", "qq_gmresdr", "qq_gmresproj", "qq_gmresdrshift", "qq_psc",
    "qq_bicgstab", "qq_fermprop", "qq_pointsource", "qq_fermprop_batch", "qq_initlagfib",
    "qq_rnds", "qq_z2source", "qq_z4source", "qq_twaverage_level0", "qq_discon_traces", "qq_bench_hsingle",
    "qq_heatbath", "qq_ctx_stream", "qq_launch_count", "qq_profile_hop", "qq_profile_hop_read",
    "qq_profile_hop_select",
    "qq_gfwrite", "qq_gfread", "qq_fpwrite", "qq_fpread", "qq_hsingle_block",
    "qq_hop_tuned_shape", "qq_net_create", "qq_net_destroy", "qq_net_nweights", "qq_net_get_weights",
    "qq_net_set_weights", "qq_net_apply", "qq_net_grad", "qq_net_train", "qq_fgmres", "qq_pionrho", "qq_twvev", "qq_twaverage", "qq_twistdiscon", "qq_average", "qq_momfacs",
    "qq_fgmresdr", "qq_fermprop_uneven",
    "qq_eigmodes", "qq_eig_destroy", "qq_eig_info", "qq_eig_vector", "qq_xigenerator", "qq_eigaverage",
    "qq_ppcoeffs", "qq_ppaverage", "qq_xipolygenerator", "qq_generalaverage", "qq_smear", "qq_mesoncorr",
    "qq_vev", "qq_discon",
]


class QQError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class qq_geom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nt", C.c_int),
                ("bc", C.c_int * 4), ("c1", C.c_double * 4), ("c2", C.c_double * 4)]


class qq_solve_info(C.Structure):
    _fields_ = [("status", C.c_int), ("itercount", C.c_int), ("mvp", C.c_int), ("ncycles", C.c_int),
                ("true_rel", C.c_double), ("seconds", C.c_double), ("nhist", C.c_int),
                ("hist", C.c_double * 1024), ("hist_mvp", C.c_int * 1024), ("nritz", C.c_int),
                ("ritz", C.c_double * 1024), ("fallback", C.c_int), ("finished_by", C.c_int),
                ("restarts", C.c_int)]


class qq_method(C.Structure):
    _fields_ = [("m", C.c_int), ("k", C.c_int), ("precision", C.c_int), ("rhs_block", C.c_int),
                ("tol", C.c_double), ("max_outer", C.c_int), ("solver", C.c_int), ("deflate", C.c_int),
                ("defl_tol", C.c_double), ("stall_window", C.c_int)]


class qq_uneven_group(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("nrhs", C.c_int), ("kappa", C.c_double * 2), ("be", C.c_void_p),
                ("bo", C.c_void_p), ("xe", C.c_void_p), ("xo", C.c_void_p),
                ("infos", C.POINTER(qq_solve_info))]


@dataclass
class SolveInfo:
    status: int
    itercount: int
    mvp: int
    ncycles: int
    true_rel: float
    seconds: float
    hist: np.ndarray
    hist_mvp: np.ndarray
    ritz: np.ndarray
    fallback: int = 0
    finished_by: int = 0
    restarts: int = 0

    @classmethod
    def from_c(cls, s: qq_solve_info) -> "SolveInfo":
        n = s.nhist
        nr = s.nritz
        r = np.array(s.ritz[: 2 * nr]).reshape(nr, 2)
        return cls(s.status, s.itercount, s.mvp, s.ncycles, s.true_rel, s.seconds,
                   np.array(s.hist[:n]), np.array(s.hist_mvp[:n]), r[:, 0] + 1j * r[:, 1], s.fallback,
                   s.finished_by, s.restarts)


_lib = None


def load_library() -> C.CDLL:
    """Load libqqcd_gpu.so, building it with nvcc first if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        from . import build as _b
        _b.build()
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    I = C.c_int
    D = C.c_double
    IP = C.POINTER(C.c_int)
    DP = C.POINTER(C.c_double)
    sig = {
        "qq_ctx_create": ([C.POINTER(qq_geom), I, C.POINTER(P)], I),
        "qq_ctx_destroy": ([P], I),
        "qq_ctx_dims": ([P, IP, IP], I),
        "qq_last_error": ([], C.c_char_p),
        "qq_set_coact": ([P, DP, DP], I),
        "qq_gauge_upload": ([P, P, I], I),
        "qq_hsingle": ([P, P, P, I, I], I),
        "qq_hdouble": ([P, P, P, I, D], I),
        "qq_hdbletm": ([P, P, P, I, DP, I], I),
        "qq_twmshift": ([P, P, P, I, DP, I], I),
        "qq_gamma5mult": ([P, P, P, I, DP, I], I),
        "qq_vecdot": ([P, P, P, DP], I),
        "qq_vecdot_noalloc": ([P, P, P, DP], I),
        "qq_defl_create": ([P, I, I, C.POINTER(P)], I),
        "qq_defl_destroy": ([P], I),
        "qq_defl_size": ([P], I),
        "qq_defl_vector": ([P, I, P], I),
        "qq_net_train_pairs": ([P, P, I, P, P, I, D, DP], I),
        "qq_gmresdr": ([P, P, P, IP, D, I, DP, I, P, C.POINTER(qq_solve_info)], I),
        "qq_gmresproj": ([P, P, P, IP, D, I, DP, I, P, C.POINTER(qq_solve_info)], I),
        "qq_gmresdrshift": ([P, P, P, I, P, IP, D, I, DP, I, P, C.POINTER(qq_solve_info)], I),
        "qq_psc": ([P, P, P, IP, D, I, DP, I, I, P, C.POINTER(qq_solve_info)], I),
        "qq_bicgstab": ([P, P, P, D, I, DP, I, I, C.POINTER(qq_solve_info)], I),
        "qq_fermprop": ([P, P, P, DP, I, D, I, IP, P, P, I, I, P, C.POINTER(qq_solve_info)], I),
        "qq_pointsource": ([P, P, P, IP, I, I], I),
        "qq_fermprop_batch": ([P, I, P, P, DP, C.POINTER(qq_method), P, P, C.POINTER(qq_solve_info)], I),
        "qq_fermprop_uneven": ([I, C.POINTER(qq_uneven_group), C.POINTER(qq_method), I, DP], I),
        "qq_initlagfib": ([I, I], I),
        "qq_rnds": ([I, DP], I),
        "qq_z2source": ([P, P, P], I),
        "qq_z4source": ([P, P, P], I),
        "qq_twaverage_level0": ([P, P, P, P, P, D, D, I, P], I),
        "qq_discon_traces": ([P, I, I, DP, C.POINTER(qq_method), D, I, P, C.POINTER(qq_solve_info)], I),
        "qq_bench_hsingle": ([P, I, I, I, I, I, DP, DP], I),
        "qq_hsingle_block": ([P, I, I, I, P, P, I, I], I),
        "qq_hop_tuned_shape": ([P, I, I, IP], I),
        "qq_net_create": ([I, IP, C.c_ulonglong, D, C.POINTER(P)], I),
        "qq_net_destroy": ([P], I),
        "qq_net_nweights": ([P], I),
        "qq_net_get_weights": ([P, DP], I),
        "qq_net_set_weights": ([P, DP], I),
        "qq_net_apply": ([P, P, P, P], I),
        "qq_net_grad": ([P, P, I, P, P, DP, DP], I),
        "qq_net_train": ([P, P, DP, I, I, D, C.c_ulonglong, DP], I),
        "qq_fgmres": ([P, P, P, P, I, D, I, DP, C.POINTER(qq_solve_info)], I),
        "qq_fgmresdr": ([P, P, P, P, IP, D, I, DP, C.POINTER(qq_solve_info)], I),
        "qq_pionrho": ([P, P, P, I, P, P, P], I),
        "qq_twvev": ([P, D, D, IP, I, I, I, I, I, P], I),
        "qq_average": ([P, P, P, P, P, D, I, I, I, P, P], I),
        "qq_momfacs": ([IP, IP, P], I),
        "qq_eigmodes": ([P, I, IP, I, DP, P, P, C.POINTER(P), IP, DP], I),
        "qq_eig_destroy": ([P], I),
        "qq_eig_info": ([P, IP, IP, IP, IP, DP, DP], I),
        "qq_eig_vector": ([P, I, I, P, P], I),
        "qq_xigenerator": ([P, P, D, DP], I),
        "qq_eigaverage": ([P, P, P, P, D, DP, I, I, P], I),
        "qq_ppcoeffs": ([P, P, P, D, I, DP], I),
        "qq_smear": ([P, P, P, P, P, D, I], I),
        "qq_mesoncorr": ([P, P, P, IP, I, P, P], I),
        "qq_ppaverage": ([P, I, DP, P, P, P, P, D, I, P], I),
        "qq_xipolygenerator": ([P, P, D, DP, DP], I),
        "qq_generalaverage": ([P, P, P, P, P, P, P, D, I, I, DP, DP, DP, DP, P], I),
        "qq_twaverage": ([P, P, P, P, P, D, D, IP, I, I, I, I, I, P], I),
        "qq_twistdiscon": ([P, I, I, DP, P, D, IP, I, I, I, I, I, P, P, P], I),
        "qq_vev": ([P, D, IP, P, P, P], I),
        "qq_discon": ([P, I, I, D, P, IP, I, I, I, P, P, P], I),
        "qq_heatbath": ([P, D, I, C.c_ulonglong, P, DP], I),
        "qq_ctx_stream": ([P, C.POINTER(P)], I),
        "qq_launch_count": ([], C.c_longlong),
        "qq_profile_hop": ([P, I], I),
        "qq_profile_hop_read": ([P, C.POINTER(C.c_longlong), DP, DP], I),
        "qq_profile_hop_select": ([P, I, I, C.POINTER(C.c_longlong), DP, DP, DP], I),
        "qq_gfwrite": ([C.c_char_p, P, I, I, IP, D, DP, DP, I, I], I),
        "qq_gfread": ([C.c_char_p, P, I, I, IP, DP, DP, DP, IP, IP], I),
        "qq_fpwrite": ([C.c_char_p, P, P, I, I, D, D, D, I, I, I, I], I),
        "qq_fpread": ([C.c_char_p, P, P, I, I, DP, DP, DP, IP, IP, IP, IP], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _check(status: int, allow_not_converged: bool = False) -> int:
    if status == QQ_OK or (allow_not_converged and status == QQ_NOT_CONVERGED):
        return status
    msg = load_library().qq_last_error().decode(errors="replace")
    raise QQError(status, msg)


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        if not (a.flags["C_CONTIGUOUS"] and a.dtype == np.float64):
            raise ValueError("reference arrays must be C-contiguous float64")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    raise TypeError(f"unsupported array type {type(a)}")


def _d2(v) -> C.Array:
    arr = (C.c_double * 2)()
    arr[0], arr[1] = float(v[0]), float(v[1])
    return arr


def _i2(v) -> C.Array:
    arr = (C.c_int * 2)()
    arr[0], arr[1] = int(v[0]), int(v[1])
    return arr


class Deflation:
    """Deflation space of GMRES-DR (replaces module ``shift`` of Q/shift.f90)."""

    def __init__(self, lat: "Lattice", nmax: int, kmax: int):
        self.lat = lat
        self._h = C.c_void_p()
        _check(lat.lib.qq_defl_create(lat._ctx, nmax, kmax, C.byref(self._h)))

    @property
    def k(self) -> int:
        return self.lat.lib.qq_defl_size(self._h)

    def vector(self, j: int, out=None):
        """Deflation vector j (0..k) as a reference-layout even half vector."""
        out = self.lat.new_half() if out is None else out
        _check(self.lat.lib.qq_defl_vector(self._h, int(j), _ptr(out)))
        return out

    def close(self):
        if self._h:
            self.lat.lib.qq_defl_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _c2(a) -> np.ndarray:
    """Complex vector as contiguous (n, 2) doubles."""
    a = np.asarray(a, complex).ravel()
    out = np.zeros((len(a), 2))
    out[:, 0], out[:, 1] = a.real, a.imag
    return out


class Eigenmodes:
    """Kept eigenmodes of M (kind 1) or of M gamma5 (kind 2) on the device
    (eigmodesofM / eigmodesofMprime, Q/disconloops.f90:1593-1937, 2573-2875)."""

    def __init__(self, lat: "Lattice", kind: int, nGMRES, ncycles: int, kappa, se=None, so=None):
        self.lat = lat
        self.kind = int(kind)
        self._h = C.c_void_p()
        g = np.ascontiguousarray(nGMRES, dtype=np.int32)
        k = np.ascontiguousarray(kappa, dtype=np.float64)
        n = C.c_int(0)
        ev = np.zeros(2 * int(nGMRES[1]))
        _check(lat.lib.qq_eigmodes(lat._ctx, self.kind, g.ctypes.data_as(C.POINTER(C.c_int)), int(ncycles),
                                   k.ctypes.data_as(C.POINTER(C.c_double)), _ptr(se) if se is not None else None,
                                   _ptr(so) if so is not None else None, C.byref(self._h), C.byref(n),
                                   ev.ctypes.data_as(C.POINTER(C.c_double))))
        self.num = n.value
        self.evals = ev[0:2 * self.num:2] + 1j * ev[1:2 * self.num:2]
        cyc, mvp = C.c_int(0), C.c_int(0)
        ritz = np.zeros(2 * int(nGMRES[1]))
        _check(lat.lib.qq_eig_info(self._h, None, None, C.byref(cyc), C.byref(mvp), None,
                                   ritz.ctypes.data_as(C.POINTER(C.c_double))))
        self.cycles, self.mvp = cyc.value, mvp.value
        self.ritz = ritz[0::2] + 1j * ritz[1::2]

    def vector(self, j: int, left: bool = False):
        """Mode j as (2,) + half_shape: the even and the odd reference-layout halves."""
        out = np.zeros((2,) + self.lat.half_shape)
        _check(self.lat.lib.qq_eig_vector(self._h, int(j), int(bool(left)), _ptr(out[0]), _ptr(out[1])))
        return out

    def xigenerator(self, kappa: float):
        """xigenerator (Q/disconloops.f90:465-838): xiinv as complex (num, 6)."""
        xi = np.zeros((max(self.num, 1), 6, 2))
        _check(self.lat.lib.qq_xigenerator(self.lat._ctx, self._h, float(kappa),
                                           xi.ctypes.data_as(C.POINTER(C.c_double))))
        return (xi[..., 0] + 1j * xi[..., 1])[:self.num]

    def eigaverage(self, ze, zo, kappa: float, scal, eigstart: int = 1, eigstep: int = 1):
        """eigaverage (Q/disconloops.f90:3239-3342) at imom = 1: (9, num, nt, 2)."""
        J = np.zeros((9, max(self.num, 1), self.lat.dims[3], 2))
        s = np.zeros((max(self.num, 1), 2))
        s[:self.num, 0] = np.real(scal)
        s[:self.num, 1] = np.imag(scal)
        _check(self.lat.lib.qq_eigaverage(self.lat._ctx, self._h, _ptr(ze), _ptr(zo), float(kappa),
                                          s.ctypes.data_as(C.POINTER(C.c_double)), int(eigstart), int(eigstep),
                                          _ptr(J)))
        return J[:, :self.num]

    def xipolygenerator(self, kappa: float, co):
        """xipolygenerator (Q/disconloops.f90:847-1584) with coefficients co (complex (8,)):
        xiinv as complex (num, 6)."""
        xi = np.zeros((max(self.num, 1), 6, 2))
        c2 = _c2(co)
        _check(self.lat.lib.qq_xipolygenerator(self.lat._ctx, self._h, float(kappa),
                                               c2.ctypes.data_as(C.POINTER(C.c_double)),
                                               xi.ctypes.data_as(C.POINTER(C.c_double))))
        return (xi[..., 0] + 1j * xi[..., 1])[:self.num]

    def close(self):
        if self._h:
            self.lat.lib.qq_eig_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Lattice:
    """One lattice (geometry, action coefficients and gauge field) on one GPU.

    bc: boundary factors (1 periodic, -1 antiperiodic, 0 fixed), the reference's
    bc(mu).  c1, c2: coact(3,1,mu) and coact(3,2,mu) (1.0 for the isotropic,
    tadpole-free actions of every configuration)."""

    def __init__(self, nx, ny, nz, nt, bc=(1, 1, 1, -1), c1=(1.0,) * 4, c2=(1.0,) * 4, device=0):
        self.lib = load_library()
        g = qq_geom(nx, ny, nz, nt, (C.c_int * 4)(*bc), (C.c_double * 4)(*c1), (C.c_double * 4)(*c2))
        self._ctx = C.c_void_p()
        _check(self.lib.qq_ctx_create(C.byref(g), device, C.byref(self._ctx)))
        nv, nt_ = C.c_int(), C.c_int()
        _check(self.lib.qq_ctx_dims(self._ctx, C.byref(nv), C.byref(nt_)))
        self.dims = (nx, ny, nz, nt)
        self.bc = tuple(bc)
        self.nvhalf, self.ntotal = nv.value, nt_.value

    # ---- shapes ----
    @property
    def half_shape(self):
        return (8, 2, 4, self.ntotal, 6)

    @property
    def gauge_shape(self):
        return (16, 2, 4, self.ntotal, 18)

    def new_half(self) -> np.ndarray:
        return np.zeros(self.half_shape)

    def close(self):
        if self._ctx:
            self.lib.qq_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- gauge ----
    def gauge_upload(self, u, recon: int = 0):
        _check(self.lib.qq_gauge_upload(self._ctx, _ptr(u), recon))

    def heatbath(self, beta=6.0, nsweeps=200, seed=13, u_out=None):
        """Generate (cold start + nsweeps heatbath sweeps) and upload a quenched SU(3)
        configuration; returns (u in reference layout or u_out, plaquette)."""
        u = np.zeros(self.gauge_shape) if u_out is None else u_out
        pl = C.c_double()
        _check(self.lib.qq_heatbath(self._ctx, float(beta), int(nsweeps), int(seed), _ptr(u), C.byref(pl)))
        return u, pl.value

    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) all calls of this lattice run on."""
        h = C.c_void_p()
        _check(self.lib.qq_ctx_stream(self._ctx, C.byref(h)))
        return h.value or 0

    def profile_hop(self, enable: bool):
        _check(self.lib.qq_profile_hop(self._ctx, int(enable)))

    def profile_hop_read(self):
        """(launches, total ms, total algorithmic bytes) of hopping kernels since enable."""
        n, ms, by = C.c_longlong(), C.c_double(), C.c_double()
        _check(self.lib.qq_profile_hop_read(self._ctx, C.byref(n), C.byref(ms), C.byref(by)))
        return n.value, ms.value, by.value

    def profile_hop_select(self, precision: int = 0, nrhs: int = 0):
        """(launches, total ms, algorithmic bytes, flops) of the profiled hopping launches
        of one spinor precision and RHS count (0: any)."""
        n, ms, by, fl = C.c_longlong(), C.c_double(), C.c_double(), C.c_double()
        _check(self.lib.qq_profile_hop_select(self._ctx, int(precision), int(nrhs), C.byref(n), C.byref(ms),
                                              C.byref(by), C.byref(fl)))
        return n.value, ms.value, by.value, fl.value

    def set_coact(self, c1, c2):
        _check(self.lib.qq_set_coact(self._ctx, (C.c_double * 4)(*c1), (C.c_double * 4)(*c2)))

    # ---- operator (Q/diracops.f90) ----
    def hsingle(self, gin, idag: int, gblclr: int, out=None):
        out = self.new_half() if out is None else out
        _check(self.lib.qq_hsingle(self._ctx, _ptr(out), _ptr(gin), idag, gblclr))
        return out

    def hop_tuned_shape(self, precision: int, nrhs: int) -> int:
        """The hopping-kernel shape the autotuner chose for this precision and RHS count."""
        v = C.c_int()
        _check(self.lib.qq_hop_tuned_shape(self._ctx, precision, nrhs, C.byref(v)))
        return v.value

    def hsingle_block(self, gin, idag: int, gblclr: int, precision: int = 32, shape: int = 0):
        """H on a stack of half vectors (shape (nrhs,) + half_shape) in reduced precision
        through one hopping-kernel shape (0 = autotuned); returns FP64 half vectors."""
        gin = np.ascontiguousarray(gin, dtype=np.float64)
        out = np.zeros_like(gin)
        _check(self.lib.qq_hsingle_block(self._ctx, precision, gin.shape[0], shape, _ptr(out), _ptr(gin),
                                         idag, gblclr))
        return out

    def hdouble(self, ge, idag: int, kappa: float, out=None):
        out = self.new_half() if out is None else out
        _check(self.lib.qq_hdouble(self._ctx, _ptr(out), _ptr(ge), idag, float(kappa)))
        return out

    def hdbletm(self, ge, idag: int, kappa, iflag: int = -1, out=None):
        out = self.new_half() if out is None else out
        _check(self.lib.qq_hdbletm(self._ctx, _ptr(out), _ptr(ge), idag, _d2(kappa), iflag))
        return out

    def twmshift(self, gwhole, idag: int, kappa, iflag: int = -1, out=None):
        out = np.zeros((2,) + self.half_shape) if out is None else out
        _check(self.lib.qq_twmshift(self._ctx, _ptr(out), _ptr(gwhole), idag, _d2(kappa), iflag))
        return out

    def gamma5mult(self, ge, idag: int, kappa, iflag: int = -1, out=None):
        """gamma5mult (Q/diracops.f90:1750-1860): -i gamma5 Hdbletm(ge) / (2 kappa mu)."""
        out = self.new_half() if out is None else out
        _check(self.lib.qq_gamma5mult(self._ctx, _ptr(out), _ptr(ge), idag, _d2(kappa), iflag))
        return out

    def vecdot(self, a, b) -> complex:
        r = (C.c_double * 2)()
        _check(self.lib.qq_vecdot(self._ctx, _ptr(a), _ptr(b), r))
        return complex(r[0], r[1])

    def vecdot_noalloc(self, a, b) -> complex:
        """vecdot of two torch CUDA tensors in the reference layout, allocating no
        device memory (qq_vecdot_noalloc)."""
        r = (C.c_double * 2)()
        _check(self.lib.qq_vecdot_noalloc(self._ctx, _ptr(a), _ptr(b), r))
        return complex(r[0], r[1])

    # ---- inverters (Q/inverters.f90) ----
    def deflation(self, nmax: int, kmax: int) -> Deflation:
        return Deflation(self, nmax, kmax)

    def gmresdr(self, phi, x, GMRES, resmax, itermin=0, kappa=(0.15, 0.0), iflag=-1, defl=None):
        info = qq_solve_info()
        st = self.lib.qq_gmresdr(self._ctx, _ptr(phi), _ptr(x), _i2(GMRES), float(resmax), itermin,
                                 _d2(kappa), iflag, defl._h if defl else None, C.byref(info))
        _check(st, allow_not_converged=True)
        return x, SolveInfo.from_c(info)

    def pionrho(self, xe, xo, idsrc: int, pion=None, rho=None, decay=None):
        """pionrho: add one propagator column's local pion, rho and decay correlators
        (length nt each) to the given arrays (new zero arrays if None)."""
        nt = self.dims[3]
        pion = np.zeros(nt) if pion is None else pion
        rho = np.zeros(nt) if rho is None else rho
        decay = np.zeros(nt) if decay is None else decay
        _check(self.lib.qq_pionrho(self._ctx, _ptr(xe), _ptr(xo), int(idsrc), _ptr(pion), _ptr(rho), _ptr(decay)))
        return pion, rho, decay

    def average(self, be, bo, xe, xo, kappa, nsub=6, nmom=5, nop=9, momfac=None):
        """average (qq_average): the Wilson loop operators of one noise at subtraction
        levels 1..nsub; momfac in numpy shape (>= 5, nmom-1, 16, 2, nvhalf).  Returns
        Jtime as an array (nop, nmom, nsub, nt, 2)."""
        J = np.zeros((nop, nmom, nsub, self.dims[3], 2))
        mf = None if momfac is None else np.ascontiguousarray(momfac, dtype=np.float64)
        _check(self.lib.qq_average(self._ctx, _ptr(be), _ptr(bo), _ptr(xe), _ptr(xo), float(kappa), int(nsub),
                                   int(nmom), int(nop), _ptr(mf) if mf is not None else None, _ptr(J)))
        return J

    def smear(self, ge, go, asmear, nsmear):
        """qq_smear: nsmear sweeps of gauge-covariant spatial smearing of a reference-layout
        pair; returns (he, ho)."""
        he, ho = self.new_half(), self.new_half()
        _check(self.lib.qq_smear(self._ctx, _ptr(he), _ptr(ho), _ptr(ge), _ptr(go), float(asmear), int(nsmear)))
        return he, ho

    def mesoncorr(self, q, src, qbar=None, channels=0):
        """qq_mesoncorr: q and qbar as (12, 2) + half_shape (column (jc-1)*4 + jd-1, even
        then odd half).  Returns corrRe, corrIm as (28, 9, 9, 9, nt) arrays (the reverse of
        the Fortran (nt, -4:4, -4:4, -4:4, 28))."""
        re = np.zeros((28, 9, 9, 9, self.dims[3]))
        im = np.zeros_like(re)
        sv = np.ascontiguousarray(src, dtype=np.int32)
        _check(self.lib.qq_mesoncorr(self._ctx, _ptr(q), _ptr(qbar) if qbar is not None else None,
                                     sv.ctypes.data_as(C.POINTER(C.c_int)), int(channels), _ptr(re), _ptr(im)))
        return re, im

    def ppcoeffs(self, be, bo, kappa, p):
        """qq_ppcoeffs: the least-squares polynomial of ppaverage* (complex (p,))."""
        co = np.zeros((p, 2))
        _check(self.lib.qq_ppcoeffs(self._ctx, _ptr(be), _ptr(bo), float(kappa), int(p),
                                    co.ctypes.data_as(C.POINTER(C.c_double))))
        return co[:, 0] + 1j * co[:, 1]

    def ppaverage(self, p, co, be, bo, xe, xo, kappa, nsub=6):
        """qq_ppaverage (ppaverage p = 5, ppaverage1 p = 8, ppaverage2 p = 11) at imom = 1:
        Jtime as (9, nsub, nt, 2)."""
        J = np.zeros((9, nsub, self.dims[3], 2))
        c2 = _c2(co)
        _check(self.lib.qq_ppaverage(self._ctx, int(p), c2.ctypes.data_as(C.POINTER(C.c_double)), _ptr(be), _ptr(bo),
                                     _ptr(xe), _ptr(xo), float(kappa), int(nsub), _ptr(J)))
        return J

    def generalaverage(self, m: "Eigenmodes", mp: "Eigenmodes", ze, zo, xe, xo, kappa, co11, co8, co5, copoly,
                       eigstart=1, eigstep=1):
        """qq_generalaverage at imom = 1: Jave as (9, 10, numEV_MAX, 6, nt, 2)."""
        ne = max(1, m.num, mp.num)
        J = np.zeros((9, 10, ne, 6, self.dims[3], 2))
        cs = [_c2(c) for c in (co11, co8, co5, copoly)]
        _check(self.lib.qq_generalaverage(self._ctx, m._h, mp._h, _ptr(ze), _ptr(zo), _ptr(xe), _ptr(xo), float(kappa),
                                          int(eigstart), int(eigstep),
                                          *[c.ctypes.data_as(C.POINTER(C.c_double)) for c in cs], _ptr(J)))
        return J

    def eigenmodes(self, kind, nGMRES, ncycles, kappa, se=None, so=None) -> Eigenmodes:
        """qq_eigmodes: kept eigenmodes of M (kind 1, from the unit source) or of M gamma5
        (kind 2, from the start vector se, so)."""
        return Eigenmodes(self, kind, nGMRES, ncycles, kappa, se, so)

    def twvev(self, kappa, delta=0.0, io=(1, 1, 1), dobndry=0, ir=1, nsub=6, nmom=5, nop=6):
        """twvev: the perturbative vacuum expectation values Jvev, as an array of shape
        (nop, nmom, 6, nt, 2) (the reverse of the Fortran (2, nt, 6, nmom, nop))."""
        J = np.zeros((nop, nmom, 6, self.dims[3], 2))
        iov = np.ascontiguousarray(io, dtype=np.int32)
        _check(self.lib.qq_twvev(self._ctx, float(kappa), float(delta), iov.ctypes.data_as(C.POINTER(C.c_int)),
                                 int(dobndry), int(ir), int(nsub), int(nmom), int(nop), _ptr(J)))
        return J

    def fgmres(self, phi, kappa, m=20, resmax=1e-10, max_cycles=200, net=None, x=None, k=0):
        """Flexible GMRES(m) -- with k > 0 flexible GMRES-DR(m, k) -- with the network
        `net` (a Net, or None) as right preconditioner, falling back to plain GMRES-DR
        if it stalls: (x, SolveInfo)."""
        x = np.zeros_like(phi) if x is None else x
        info = qq_solve_info()
        h = net._h if net is not None else None
        if k:
            st = self.lib.qq_fgmresdr(self._ctx, h, _ptr(phi), _ptr(x), _i2((m, k)), float(resmax),
                                      int(max_cycles), _d2(kappa), C.byref(info))
        else:
            st = self.lib.qq_fgmres(self._ctx, h, _ptr(phi), _ptr(x), int(m), float(resmax), int(max_cycles),
                                    _d2(kappa), C.byref(info))
        _check(st, allow_not_converged=True)
        return x, SolveInfo.from_c(info)

    def gmresproj(self, b, x, GMRES, resmax, itermin=0, kappa=(0.15, 0.0), iflag=-1, defl=None):
        info = qq_solve_info()
        st = self.lib.qq_gmresproj(self._ctx, _ptr(b), _ptr(x), _i2(GMRES), float(resmax), itermin,
                                   _d2(kappa), iflag, defl._h, C.byref(info))
        _check(st, allow_not_converged=True)
        return x, SolveInfo.from_c(info)

    def gmresdrshift(self, b, sigma, GMRES, resmax, itermin=0, kappa=(0.15, 0.01), iflag=-1):
        """gmresdrshift (Q/inverters.f90:6041-7179): solutions of (A - sigma_s) x_s = b for
        every shift, A = gamma5mult, from one deflated Krylov space.  Returns
        (x[nshifts, ...], resid[nshifts] (absolute), SolveInfo)."""
        sig = np.ascontiguousarray(sigma, dtype=np.float64)
        ns = int(sig.shape[0])
        x = np.zeros((ns,) + self.half_shape)
        resid = np.zeros(ns)
        info = qq_solve_info()
        st = self.lib.qq_gmresdrshift(self._ctx, _ptr(b), _ptr(x), ns, _ptr(sig), _i2(GMRES), float(resmax),
                                      itermin, _d2(kappa), iflag, _ptr(resid), C.byref(info))
        _check(st, allow_not_converged=True)
        return x, resid, SolveInfo.from_c(info)

    def psc(self, b, x, GMRES, resmax, itermin=0, kappa=(0.15, 0.0), iflag=-1, isignal=1, defl=None):
        info = qq_solve_info()
        st = self.lib.qq_psc(self._ctx, _ptr(b), _ptr(x), _i2(GMRES), float(resmax), itermin,
                             _d2(kappa), iflag, isignal, defl._h, C.byref(info))
        _check(st, allow_not_converged=True)
        return x, SolveInfo.from_c(info)

    def bicgstab(self, phi, x, resmax, itermin=0, kappa=(0.15, 0.0), iflag=-1, maxiter=0):
        info = qq_solve_info()
        st = self.lib.qq_bicgstab(self._ctx, _ptr(phi), _ptr(x), float(resmax), itermin, _d2(kappa),
                                  iflag, maxiter, C.byref(info))
        _check(st, allow_not_converged=True)
        return x, SolveInfo.from_c(info)

    # ---- propagators (Q/quark.f90) ----
    def fermprop(self, be, bo, kappa, inverter=5, resmax=1e-10, itermin=0, nGMRES=(30, 10),
                 ntmqcd=0, isignal=1, defl=None, xe=None, xo=None):
        xe = self.new_half() if xe is None else xe
        xo = self.new_half() if xo is None else xo
        info = qq_solve_info()
        st = self.lib.qq_fermprop(self._ctx, _ptr(be), _ptr(bo), _d2(kappa), inverter, float(resmax),
                                  itermin, _i2(nGMRES), _ptr(xe), _ptr(xo), ntmqcd, isignal,
                                  defl._h if defl else None, C.byref(info))
        _check(st, allow_not_converged=True)
        return xe, xo, SolveInfo.from_c(info)

    def pointsource(self, src, icsrc: int, idsrc: int):
        be, bo = self.new_half(), self.new_half()
        _check(self.lib.qq_pointsource(self._ctx, _ptr(be), _ptr(bo), (C.c_int * 4)(*src), icsrc, idsrc))
        return be, bo

    def fermprop_batch(self, be, bo, kappa, m=60, k=20, precision=32, rhs_block=12, tol=1e-10,
                       max_outer=0, solver=1, deflate=1, defl_tol=1e-5, xe=None, xo=None, stall_window=0):
        """Batched propagators (qq_fermprop_batch): be, bo of shape (nrhs,) + half_shape,
        numpy (host) or torch CUDA tensors.  solver=0 is the reference's plain FP64
        GMRES-DR(m,k) per right-hand side; solver=1 the deflated batched BiCGStab, whose
        right-hand sides that break down, stall for stall_window iterations (0: 2000) or
        run out of iterations are finished by plain FP64 GMRES-DR (info.fallback)."""
        nrhs = be.shape[0]
        if xe is None:
            xe = np.zeros(be.shape) if isinstance(be, np.ndarray) else be.new_zeros(be.shape)
        if xo is None:
            xo = np.zeros(bo.shape) if isinstance(bo, np.ndarray) else bo.new_zeros(bo.shape)
        infos = (qq_solve_info * nrhs)()
        meth = qq_method(m, k, precision, rhs_block, tol, max_outer, solver, deflate, defl_tol, stall_window)
        st = self.lib.qq_fermprop_batch(self._ctx, nrhs, _ptr(be), _ptr(bo), _d2(kappa), C.byref(meth),
                                        _ptr(xe), _ptr(xo), infos)
        _check(st, allow_not_converged=True)
        return xe, xo, [SolveInfo.from_c(i) for i in infos]

    # ---- noise sources and traces (Q/disconloops.f90) ----
    def z2source(self):
        be, bo = self.new_half(), self.new_half()
        _check(self.lib.qq_z2source(self._ctx, _ptr(be), _ptr(bo)))
        return be, bo

    def z4source(self):
        be, bo = self.new_half(), self.new_half()
        _check(self.lib.qq_z4source(self._ctx, _ptr(be), _ptr(bo)))
        return be, bo

    def discon_traces(self, noise_kind: int, nnoise: int, kappa, solver: int = 1, m: int = 60, k: int = 20,
                      precision: int = 32, rhs_block: int = 12, tol: float = 1e-10, max_outer: int = 0,
                      deflate: int = 0, defl_tol: float = 1e-5, delta: float = 0.0, dobndry: int = 0):
        """Noise-averaged level-0 loop traces (qq_discon_traces): J[iop, t, re/im] and the
        per-noise solve reports.  Call initlagfib first, as the reference does."""
        J = np.zeros((6, self.dims[3], 2))
        infos = (qq_solve_info * nnoise)()
        meth = qq_method(m, k, precision, rhs_block, tol, max_outer, solver, deflate, defl_tol)
        st = self.lib.qq_discon_traces(self._ctx, int(noise_kind), int(nnoise), _d2(kappa), C.byref(meth),
                                       float(delta), int(dobndry), _ptr(J), infos)
        _check(st, allow_not_converged=True)
        return J, [SolveInfo.from_c(i) for i in infos]

    def twaverage(self, be, bo, xe, xo, kappa: float = 0.0, delta: float = 0.0, io=(1, 1, 1), dobndry: int = 0,
                  nsub: int = 0, nmom: int = 5, nop: int = 6, ir: int = 1):
        """twAverage of one noise (qq_twaverage): Jave as an array (nop, nmom, 6, nt, 2)."""
        J = np.zeros((nop, nmom, 6, self.dims[3], 2))
        iov = np.ascontiguousarray(io, dtype=np.int32)
        _check(self.lib.qq_twaverage(self._ctx, _ptr(be), _ptr(bo), _ptr(xe), _ptr(xo), float(kappa), float(delta),
                                     iov.ctypes.data_as(C.POINTER(C.c_int)), int(dobndry), int(ir), int(nsub),
                                     int(nmom), int(nop), _ptr(J)))
        return J

    def twistdiscon(self, noise_kind: int, nnoise: int, kappa, nsub: int = 6, nmom: int = 5, nop: int = 6,
                    io=(1, 1, 1), delta: float = 0.0, dobndry: int = 0, ir: int = 1, solver: int = 0, m: int = 30,
                    k: int = 10,
                    precision: int = 32, rhs_block: int = 12, tol: float = 1e-10, max_outer: int = 0,
                    deflate: int = 0, defl_tol: float = 1e-5, per_noise: bool = False):
        """twistdiscon (qq_twistdiscon): Jtotal as an array (nop, nmom, 6, nt, 2) and the
        per-noise solve reports; with per_noise also every noise's values as an array
        (nnoise, nop, nmom, 6, nt, 2).  Call initlagfib first, as the reference does."""
        J = np.zeros((nop, nmom, 6, self.dims[3], 2))
        Jn = np.zeros((nnoise, nop, nmom, 6, self.dims[3], 2)) if per_noise else None
        infos = (qq_solve_info * nnoise)()
        meth = qq_method(m, k, precision, rhs_block, tol, max_outer, solver, deflate, defl_tol)
        iov = np.ascontiguousarray(io, dtype=np.int32)
        st = self.lib.qq_twistdiscon(self._ctx, int(noise_kind), int(nnoise), _d2(kappa), C.byref(meth),
                                     float(delta), iov.ctypes.data_as(C.POINTER(C.c_int)), int(dobndry), int(ir),
                                     int(nsub), int(nmom), int(nop), _ptr(J), _ptr(Jn) if per_noise else None,
                                     infos)
        _check(st, allow_not_converged=True)
        if per_noise:
            return J, [SolveInfo.from_c(i) for i in infos], Jn
        return J, [SolveInfo.from_c(i) for i in infos]

    def vev(self, kappa: float, io=(1, 1, 1)):
        """vev (qq_vev): the Wilson loop driver's perturbative vacuum values on the uploaded
        gauge field.  Returns (Jvev as an array (5 op, 5 momenta, nt, 2), the average
        plaquette, <psibar psi>)."""
        J = np.zeros((5, 5, self.dims[3], 2))
        plaq = np.zeros(1)
        psi = np.zeros(1)
        iov = np.ascontiguousarray(io, dtype=np.int32)
        _check(self.lib.qq_vev(self._ctx, float(kappa), iov.ctypes.data_as(C.POINTER(C.c_int)), _ptr(J),
                               _ptr(plaq), _ptr(psi)))
        return J, float(plaq[0]), float(psi[0])

    def discon(self, noise_kind: int, nnoise: int, kappa: float, nsub: int = 6, nmom: int = 5, nop: int = 5,
               io=(1, 1, 1), solver: int = 0, m: int = 30, k: int = 10, precision: int = 32, rhs_block: int = 12,
               tol: float = 1e-10, max_outer: int = 0, deflate: int = 0, defl_tol: float = 1e-5):
        """discon (qq_discon), one run of the Wilson loop driver: Jtotal as an array (nop, nmom,
        nsub, nt, 2), the vev's Jvev (5, 5, nt, 2) and the per-noise solve reports.  Call
        initlagfib first, as the reference does."""
        J = np.zeros((nop, nmom, nsub, self.dims[3], 2))
        Jv = np.zeros((5, 5, self.dims[3], 2))
        infos = (qq_solve_info * nnoise)()
        meth = qq_method(m, k, precision, rhs_block, tol, max_outer, solver, deflate, defl_tol)
        iov = np.ascontiguousarray(io, dtype=np.int32)
        st = self.lib.qq_discon(self._ctx, int(noise_kind), int(nnoise), float(kappa), C.byref(meth),
                                iov.ctypes.data_as(C.POINTER(C.c_int)), int(nsub), int(nmom), int(nop), _ptr(J),
                                _ptr(Jv), infos)
        _check(st, allow_not_converged=True)
        return J, Jv, [SolveInfo.from_c(i) for i in infos]

    def twaverage_level0(self, be, bo, xe, xo, kappa: float, delta: float = 0.0, dobndry: int = 0):
        """Level-0 loop traces of one noise (qq_twaverage_level0): J[iop, t, re/im]."""
        J = np.zeros((6, self.dims[3], 2))
        _check(self.lib.qq_twaverage_level0(self._ctx, _ptr(be), _ptr(bo), _ptr(xe), _ptr(xo),
                                            float(kappa), float(delta), int(dobndry), _ptr(J)))
        return J


    def bench_hsingle(self, precision=64, nrhs=1, niter=20, flush_l2=True, tps=0):
        """Mean kernel time (ms) and algorithmic bytes of one hopping-term launch."""
        ms, by = C.c_double(), C.c_double()
        _check(self.lib.qq_bench_hsingle(self._ctx, precision, nrhs, tps, niter, int(flush_l2),
                                         C.byref(ms), C.byref(by)))
        return ms.value, by.value


class Net:
    """The learned preconditioner's network (qq_net_*): linear gauge-covariant
    parallel-transport convolution layers from 4 spin channels to 4, trained on the GPU
    to approximate the inverse of Hdbletm."""

    def __init__(self, channels=(4, 8, 8, 4), seed: int = 1, scale: float = 1.0):
        self.lib = load_library()
        self._h = C.c_void_p()
        arr = (C.c_int * len(channels))(*channels)
        _check(self.lib.qq_net_create(len(channels) - 1, arr, int(seed), float(scale), C.byref(self._h)))
        self.channels = tuple(channels)

    @property
    def nweights(self) -> int:
        return int(self.lib.qq_net_nweights(self._h))

    def get_weights(self) -> np.ndarray:
        w = np.zeros(2 * self.nweights)
        _check(self.lib.qq_net_get_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_double))))
        return w[0::2] + 1j * w[1::2]

    def set_weights(self, w) -> None:
        a = np.zeros(2 * self.nweights)
        a[0::2], a[1::2] = np.real(w), np.imag(w)
        _check(self.lib.qq_net_set_weights(self._h, a.ctypes.data_as(C.POINTER(C.c_double))))

    def apply(self, lat, gin):
        out = lat.new_half()
        _check(self.lib.qq_net_apply(lat._ctx, self._h, _ptr(gin), _ptr(out)))
        return out

    def loss_grad(self, lat, b, x):
        """Loss and dl/d conj(W) over pairs b[i], x[i] (stacks of half vectors)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        loss = C.c_double()
        g = np.zeros(2 * self.nweights)
        _check(self.lib.qq_net_grad(lat._ctx, self._h, b.shape[0], _ptr(b), _ptr(x), C.byref(loss),
                                    g.ctypes.data_as(C.POINTER(C.c_double))))
        return loss.value, g[0::2] + 1j * g[1::2]

    def train(self, lat, kappa, nsamples=4, nsteps=100, lr=1e-3, seed=1):
        """Adam steps on pairs (Hdbletm x, x) with Gaussian x; the loss before each step."""
        losses = np.zeros(max(nsteps, 1))
        _check(self.lib.qq_net_train(lat._ctx, self._h, _d2(kappa), int(nsamples), int(nsteps), float(lr),
                                     int(seed), losses.ctypes.data_as(C.POINTER(C.c_double))))
        return losses[:nsteps]

    def train_pairs(self, lat, b, x, nsteps=100, lr=1e-3):
        """Adam steps on the caller's pairs: sources b and targets x (arrays of shape
        (n,) + half_shape), the network learning N(b) = x; the loss before each step."""
        losses = np.zeros(max(nsteps, 1))
        _check(self.lib.qq_net_train_pairs(lat._ctx, self._h, int(b.shape[0]), _ptr(b), _ptr(x), int(nsteps),
                                           float(lr), losses.ctypes.data_as(C.POINTER(C.c_double))))
        return losses[:nsteps]

    def close(self) -> None:
        if self._h:
            self.lib.qq_net_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def launch_count() -> int:
    """Kernels launched by the library in this process so far."""
    return int(load_library().qq_launch_count())


def momfacs(dims, io=(1, 1, 1)) -> np.ndarray:
    """momfacs (qq_momfacs, host only): the Wilson driver's momentum factors as numpy
    shape (5, 4, 16, 2, nvhalf), the reverse of the Fortran (nvhalf, 2, 16, 4, 5)."""
    nv = dims[0] * dims[1] * dims[2] * dims[3] // 32
    mf = np.zeros((5, 4, 16, 2, nv))
    d = np.ascontiguousarray(dims, dtype=np.int32)
    o = np.ascontiguousarray(io, dtype=np.int32)
    _check(load_library().qq_momfacs(d.ctypes.data_as(C.POINTER(C.c_int)), o.ctypes.data_as(C.POINTER(C.c_int)),
                                     _ptr(mf)))
    return mf


def fermprop_uneven(groups, m=60, k=20, precision=32, rhs_block=12, tol=1e-10, max_outer=0, solver=1,
                    deflate=0, defl_tol=1e-5, concurrent=True, stall_window=0):
    """Uneven batch (qq_fermprop_uneven): groups is a list of (lattice, be, bo, kappa),
    be/bo of shape (nrhs,) + that lattice's half_shape, numpy or torch CUDA tensors.
    Each group is solved as Lattice.fermprop_batch solves it; with concurrent=True the
    lattices run side by side on their own streams.  Returns ([(xe, xo, infos)] per
    group, wall seconds of the call)."""
    n = len(groups)
    arr = (qq_uneven_group * n)()
    keep = []
    for i, (lat, be, bo, kappa) in enumerate(groups):
        nrhs = be.shape[0]
        xe = np.zeros(be.shape) if isinstance(be, np.ndarray) else be.new_zeros(be.shape)
        xo = np.zeros(bo.shape) if isinstance(bo, np.ndarray) else bo.new_zeros(bo.shape)
        infos = (qq_solve_info * nrhs)()
        arr[i] = qq_uneven_group(lat._ctx.value, nrhs, (C.c_double * 2)(*kappa), _ptr(be), _ptr(bo), _ptr(xe),
                                 _ptr(xo), C.cast(infos, C.POINTER(qq_solve_info)))
        keep.append((xe, xo, infos))
    meth = qq_method(m, k, precision, rhs_block, tol, max_outer, solver, deflate, defl_tol, stall_window)
    secs = C.c_double(0.0)
    _check(load_library().qq_fermprop_uneven(n, arr, C.byref(meth), int(bool(concurrent)), C.byref(secs)),
           allow_not_converged=True)
    return [(xe, xo, [SolveInfo.from_c(i) for i in infos]) for xe, xo, infos in keep], secs.value


def initlagfib(myid: int, iseed: int):
    _check(load_library().qq_initlagfib(myid, iseed))


def rnds(m: int) -> np.ndarray:
    out = np.zeros(m)
    _check(load_library().qq_rnds(m, out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


# ---- file formats of the reference (G/gaugetools.f90 GFwrite/GFread, Q/quark.f90 FPwrite/FPread)
def gfwrite(path, u: np.ndarray, nvhalf: int, gaction=(1, 1, 1, 1), beta=6.0, alat=(1.0,) * 4, tad=(1.0,) * 4,
            icfgsave=1, myid=0):
    """Write a gauge configuration (re-unitarises u in place, as GFwrite)."""
    ntotal = u.shape[3]
    _check(load_library().qq_gfwrite(str(path).encode(), _ptr(u), nvhalf, ntotal, (C.c_int * 4)(*gaction),
                                     float(beta), (C.c_double * 4)(*alat), (C.c_double * 4)(*tad),
                                     int(icfgsave), int(myid)))


def gfread(path, nvhalf: int, ntotal: int):
    """Read a gauge configuration: (u, header dict)."""
    u = np.zeros((16, 2, 4, ntotal, 18))
    ga, al, td = (C.c_int * 4)(), (C.c_double * 4)(), (C.c_double * 4)()
    beta, icfg, myid = C.c_double(), C.c_int(), C.c_int()
    _check(load_library().qq_gfread(str(path).encode(), _ptr(u), nvhalf, ntotal, ga, C.byref(beta), al, td,
                                    C.byref(icfg), C.byref(myid)))
    return u, dict(gaction=tuple(ga), beta=beta.value, alat=tuple(al), tad=tuple(td), icfgsave=icfg.value,
                   myid=myid.value)


def fpwrite(path, xe: np.ndarray, xo: np.ndarray, nvhalf: int, kappa=0.0, tmqcd=0.0, cSW=0.0, icsrc=1, idsrc=1,
            icfg=1, myid=0):
    """Write a propagator (xe: gblclr 1 half, xo: gblclr 2 half)."""
    _check(load_library().qq_fpwrite(str(path).encode(), _ptr(xe), _ptr(xo), nvhalf, xe.shape[3], float(kappa),
                                     float(tmqcd), float(cSW), int(icsrc), int(idsrc), int(icfg), int(myid)))


def fpread(path, nvhalf: int, ntotal: int):
    """Read a propagator: (xe, xo, header dict)."""
    xe = np.zeros((8, 2, 4, ntotal, 6))
    xo = np.zeros((8, 2, 4, ntotal, 6))
    k, t, c = C.c_double(), C.c_double(), C.c_double()
    ic, idd, cf, my = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    _check(load_library().qq_fpread(str(path).encode(), _ptr(xe), _ptr(xo), nvhalf, ntotal, C.byref(k), C.byref(t),
                                    C.byref(c), C.byref(ic), C.byref(idd), C.byref(cf), C.byref(my)))
    return xe, xo, dict(kappa=k.value, tmqcd=t.value, cSW=c.value, icsrc=ic.value, idsrc=idd.value,
                        icfg=cf.value, myid=my.value)
