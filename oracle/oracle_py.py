"""ctypes loader for the CPU oracle (TEST INFRASTRUCTURE: GPU results are checked against it).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.  It mirrors the reference routine names (``DFDX_sym`` ...) on
numpy arrays in the reference layout F(My,Mz,Mx[,n]); a numpy array of shape
(Mx, Mz, My) in C order has exactly that memory layout.

Parity status: unpinned by the reference's own tests (none exist, and the
Fortran reference cannot be built here); see st_oracle.h.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liborc_st.so")

sys.path.insert(0, os.path.dirname(_HERE))
from shock_turbulence_b200.params import StParams, StRadialParams, default_params  # noqa: E402

_dp = ctypes.POINTER(ctypes.c_double)


def build(force=False):
    """Compile the oracle with its Makefile (make rebuilds it when a source
    is newer than the library)."""
    args = ["make", "-s", "-C", _HERE, "liborc_st.so"]
    if force:
        args.insert(1, "-B")
    try:
        subprocess.check_call(args)
    except (OSError, subprocess.CalledProcessError):
        if not os.path.exists(_LIB):
            raise
    return _LIB


def _load():
    build()
    lib = ctypes.CDLL(_LIB)
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = [ctypes.POINTER(StParams)]
    lib.orc_destroy.argtypes = [ctypes.c_void_p]
    lib.orc_compute_tstep.restype = ctypes.c_double
    lib.orc_get_tstep.restype = ctypes.c_double
    lib.orc_set_tstep.argtypes = [ctypes.c_void_p, ctypes.c_double]
    lib.orc_dfd.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int,
                            ctypes.c_double]
    lib.orc_d2fd2.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int]
    lib.orc_filter.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp]
    lib.orc_gauss.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
    lib.orc_compact_filter.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
    lib.orc_gaussian_filter.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
    lib.orc_bc_rhs.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_double]
    lib.orc_compute_tstep.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_double, ctypes.c_int]
    lib.orc_get_common.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp]
    lib.orc_set_common.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp]
    lib.orc_tridiagonal.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.orc_pentadiagonal.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int]
    lib.orc_set_threads.argtypes = [ctypes.c_int]
    lib.orc_compute_grad.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
    lib.orc_shell_count.argtypes = [ctypes.c_void_p]
    lib.orc_compute_srm_stats.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
    lib.orc_shock_surface.argtypes = [ctypes.c_void_p, _dp, _dp]
    lib.orc_make_padded_arrays.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
    lib.orc_graph_bytes.restype = ctypes.c_double
    lib.orc_graph_bytes.argtypes = []
    lib.orc_graph_bytes_reset.argtypes = []
    rp = ctypes.POINTER(StRadialParams)
    ci, cd = ctypes.c_int, ctypes.c_double
    lib.orc_rad_radius.argtypes = [ci, cd, _dp]
    lib.orc_rad_dfdx.argtypes = [ci, cd, _dp, _dp, ci, cd]
    lib.orc_rad_d2fdx2.argtypes = [ci, cd, _dp, _dp, _dp, ci]
    lib.orc_rad_filter.argtypes = [ci, _dp, _dp]
    lib.orc_rad_gauss.argtypes = [ci, _dp, _dp]
    lib.orc_rad_rhs.argtypes = [rp, ci, cd, _dp, _dp]
    lib.orc_rad_compute_hyper.argtypes = [rp, ci, cd, _dp, _dp]
    lib.orc_rad_hyper_rhs.argtypes = [rp, ci, cd, _dp, _dp, _dp]
    lib.orc_rad_tstep.argtypes = [rp, ci, cd, _dp, _dp, _dp, _dp]
    lib.orc_rad_tstep.restype = cd
    lib.orc_rad_step.argtypes = [rp, ci, cd, _dp, _dp, _dp, ctypes.POINTER(ci)]
    lib.orc_rad_step.restype = cd
    lib.orc_rad_batch.argtypes = [rp, ci, ctypes.POINTER(ci), ctypes.POINTER(ctypes.c_longlong),
                                  _dp, _dp, _dp, _dp, ctypes.POINTER(ci), ci]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "oracle needs C-contiguous float64"
    return a.ctypes.data_as(_dp)


def graph_bytes(reset=False):
    """Interface bytes of the reference operator calls made since the last
    reset (DF*, D2F*2, filter and Gaussian passes, stage updates)."""
    v = lib().orc_graph_bytes()
    if reset:
        lib().orc_graph_bytes_reset()
    return v


def set_threads(n):
    lib().orc_set_threads(int(n))


def tridiagonal(A, B, C, R, nper=0):
    """tridiagonal(A1,B1,C1,R,n,lot,nper) on arrays of shape (n, lot); R overwritten."""
    n, lot = R.shape
    lib().orc_tridiagonal(_p(A), _p(B), _p(C), _p(R), n, lot, nper)


def pentadiagonal(A, B, C, D, E, R, nper=0):
    n, lot = R.shape
    lib().orc_pentadiagonal(_p(A), _p(B), _p(C), _p(D), _p(E), _p(R), n, lot, nper)


class Oracle:
    """One oracle context: the COMMON blocks of the reference plus its LHS."""

    def __init__(self, params=None, **kw):
        if params is None:
            params = default_params(**kw)
        self.params = params
        self.shape = (params.nx, params.nz, params.ny)   # (Mx, Mz, My) C order = F(My,Mz,Mx)
        self._c = lib().orc_create(ctypes.byref(params))

    def __del__(self):
        if getattr(self, "_c", None):
            lib().orc_destroy(self._c)
            self._c = None

    def field(self, n=None):
        return np.zeros(self.shape if n is None else (n,) + self.shape)

    # --- state ---------------------------------------------------------
    def set_state(self, Q, Y):
        lib().orc_set_state(ctypes.c_void_p(self._c), _p(np.ascontiguousarray(Q)),
                            None if Y is None else _p(np.ascontiguousarray(Y)))

    def get_state(self):
        Q, Y = self.field(5), self.field()
        lib().orc_get_state(ctypes.c_void_p(self._c), _p(Q), _p(Y))
        return Q, Y

    def set_tstep(self, t):
        lib().orc_set_tstep(self._c, float(t))

    def get_tstep(self):
        return lib().orc_get_tstep(ctypes.c_void_p(self._c))

    def get_common(self, name):
        n = 5 if name in ("dQ", "QW") else None
        out = self.field(n)
        if lib().orc_get_common(self._c, name.encode(), _p(out)) != 0:
            raise KeyError(name)
        return out

    def set_common(self, name, arr):
        if lib().orc_set_common(self._c, name.encode(), _p(np.ascontiguousarray(arr))) != 0:
            raise KeyError(name)

    # --- operators (reference names) -----------------------------------
    def dfd(self, d, asym, F, dF, iadd, cadd):
        lib().orc_dfd(self._c, d, asym, _p(F), _p(dF), iadd, float(cadd))

    def d2fd2(self, d, asym, F, dF, d2F, iadd):
        lib().orc_d2fd2(self._c, d, asym, _p(F), _p(dF), _p(d2F), iadd)

    def filter(self, d, asym, F, F0):
        lib().orc_filter(self._c, d, asym, _p(F), _p(F0))

    def gauss(self, d, F, Fg):
        lib().orc_gauss(self._c, d, _p(F), _p(Fg))

    def compact_filter(self, F, F0, nvar):
        lib().orc_compact_filter(self._c, _p(F), _p(F0), nvar)

    def gaussian_filter(self, F, Fg, nvar):
        lib().orc_gaussian_filter(self._c, _p(F), _p(Fg), nvar)

    def compute_gamma(self, Y):
        lib().orc_compute_gamma(ctypes.c_void_p(self._c), _p(Y))

    def rhs(self, Q, Qrhs, Y=None):
        lib().orc_rhs(ctypes.c_void_p(self._c), _p(Q), _p(Qrhs), _p(Y))

    def compute_hyper(self, Q, Y=None):
        lib().orc_compute_hyper(ctypes.c_void_p(self._c), _p(Q), _p(Y))

    def hyper_rhs(self, Q, Qrhs, Y=None):
        lib().orc_hyper_rhs(ctypes.c_void_p(self._c), _p(Q), _p(Qrhs), _p(Y))

    def species_rhs(self, Q, Qrhs, Y, Yrhs):
        lib().orc_species_rhs(ctypes.c_void_p(self._c), _p(Q), _p(Qrhs), _p(Y), _p(Yrhs))

    def bc_rhs(self, Q, Qrhs, Y, Yrhs, time=0.0):
        lib().orc_bc_rhs(self._c, _p(Q), _p(Qrhs), _p(Y), _p(Yrhs), float(time))

    def sponge_forcing(self, Q, Qrhs, Y, Yrhs):
        lib().orc_sponge_forcing(ctypes.c_void_p(self._c), _p(Q), _p(Qrhs), _p(Y), _p(Yrhs))

    def fix_pressure(self, Q, Y=None):
        lib().orc_fix_pressure(ctypes.c_void_p(self._c), _p(Q), _p(Y))

    def compute_cfl(self, Q):
        a, b = ctypes.c_double(), ctypes.c_double()
        lib().orc_compute_cfl(ctypes.c_void_p(self._c), _p(Q), ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def compute_tstep(self, Q, Y, cfl_resv, step):
        return lib().orc_compute_tstep(self._c, _p(Q), _p(Y), float(cfl_resv), int(step))

    def lddrk4(self, time=0.0, step=0):
        t, s = ctypes.c_double(time), ctypes.c_int(step)
        lib().orc_lddrk4(ctypes.c_void_p(self._c), ctypes.byref(t), ctypes.byref(s))
        return t.value, s.value

    def step(self, time=0.0, step=0):
        t, s = ctypes.c_double(time), ctypes.c_int(step)
        lib().orc_step(ctypes.c_void_p(self._c), ctypes.byref(t), ctypes.byref(s))
        return t.value, s.value

    def monitors(self):
        out = np.zeros(10)
        lib().orc_get_monitors(ctypes.c_void_p(self._c), _p(out))
        return out

    # Output-side diagnostics (src/grad_sym.f, pproc/pproc_mf.f, src/shock.f)
    def compute_grad(self):
        G = np.zeros((4,) + self.shape)
        a, b = np.zeros(1), np.zeros(1)
        lib().orc_compute_grad(ctypes.c_void_p(self._c), _p(G), _p(a), _p(b))
        return G, float(a[0]), float(b[0])

    def make_padded_arrays(self, Grad):
        """MakePaddedArrays (src/vis_silo_mf.f:440-689): W (11, Mx+1, Mz+1,
        My+1) and the padded coordinates xx, yy, zz."""
        nx, nz, ny = self.shape
        G = np.ascontiguousarray(Grad, dtype=np.float64)
        W = np.zeros((11, nx + 1, nz + 1, ny + 1))
        xx, yy, zz = np.zeros(nx + 1), np.zeros(ny + 1), np.zeros(nz + 1)
        lib().orc_make_padded_arrays(ctypes.c_void_p(self._c), _p(G), _p(W), _p(xx), _p(yy), _p(zz))
        return W, xx, yy, zz

    def compute_srm_stats(self):
        na = lib().orc_shell_count(ctypes.c_void_p(self._c))
        h, t, ur, ya = np.zeros(1), np.zeros(1), np.zeros(na), np.zeros(na)
        lib().orc_compute_srm_stats(ctypes.c_void_p(self._c), _p(h), _p(t), _p(ur), _p(ya))
        return float(h[0]), float(t[0]), ur, ya

    def shock_surface(self):
        a, b = np.zeros(1), np.zeros(1)
        lib().orc_shock_surface(ctypes.c_void_p(self._c), _p(a), _p(b))
        return float(a[0]), float(b[0])


# ---- 1-D spherical-radial family (st_oracle_radial.c) ---------------------
class Radial:
    """Line operators and steps of the radial family on numpy arrays; Q of one
    problem is an array (3, n) = (u_r, rho, s), hyp (2, n) = (beta, visc)."""

    def __init__(self, params):
        self.p = params

    def radius(self, n, x_leng):
        r = np.zeros(n)
        lib().orc_rad_radius(n, float(x_leng), _p(r))
        return r

    def dfdx(self, x_leng, F, dF, iadd, cadd):
        lib().orc_rad_dfdx(F.size, float(x_leng), _p(F), _p(dF), int(iadd), float(cadd))

    def d2fdx2(self, x_leng, F, dF, d2F, iadd):
        lib().orc_rad_d2fdx2(F.size, float(x_leng), _p(F), _p(dF), _p(d2F), int(iadd))

    def filter(self, F, F0):
        lib().orc_rad_filter(F.size, _p(F), _p(F0))

    def gauss(self, F, Fg):
        lib().orc_rad_gauss(F.size, _p(F), _p(Fg))

    def rhs(self, x_leng, Q, Qrhs):
        lib().orc_rad_rhs(ctypes.byref(self.p), Q.shape[1], float(x_leng), _p(Q), _p(Qrhs))

    def compute_hyper(self, x_leng, Q, hyp):
        lib().orc_rad_compute_hyper(ctypes.byref(self.p), Q.shape[1], float(x_leng), _p(Q), _p(hyp))

    def hyper_rhs(self, x_leng, Q, Qrhs, hyp):
        lib().orc_rad_hyper_rhs(ctypes.byref(self.p), Q.shape[1], float(x_leng), _p(Q), _p(Qrhs), _p(hyp))

    def tstep(self, x_leng, Q, hyp):
        a, b = ctypes.c_double(), ctypes.c_double()
        dt = lib().orc_rad_tstep(ctypes.byref(self.p), Q.shape[1], float(x_leng), _p(Q), _p(hyp),
                                 ctypes.byref(a), ctypes.byref(b))
        return dt, a.value, b.value

    def step(self, x_leng, Q, hyp, time, step):
        t, s = ctypes.c_double(time), ctypes.c_int(step)
        lib().orc_rad_step(ctypes.byref(self.p), Q.shape[1], float(x_leng), _p(Q), _p(hyp), ctypes.byref(t),
                           ctypes.byref(s))
        return t.value, s.value

    def batch(self, lengths, x_leng, Q, hyp, time, step, nsteps):
        """nsteps steps of every packed problem (Q: 3*sum(n), hyp: 2*sum(n))."""
        n = np.ascontiguousarray(lengths, dtype=np.int32)
        off = np.zeros(len(n), dtype=np.int64)
        off[1:] = np.cumsum(n)[:-1]
        xl = np.ascontiguousarray(x_leng, dtype=np.float64)
        lib().orc_rad_batch(ctypes.byref(self.p), len(n), n.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                            off.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _p(xl), _p(Q), _p(hyp),
                            _p(time), step.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(nsteps))
