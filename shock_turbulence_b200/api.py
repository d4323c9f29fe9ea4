"""Host-side mirror of the reference's subroutine interface over the C ABI.

Method names and argument meanings follow the Fortran routines
(``DFDX_sym(F, dF, iadd, cadd)``, ``RHS(Q, Qrhs, Y)``, ``LDDRK4(time, step)``
...).  Arrays are numpy float64 arrays or torch float64 tensors (host or
CUDA) in the reference layout F(My,Mz,Mx[,n]), i.e. C-order shape
([n,] Mx, Mz, My).  Outputs are written in place, as in the reference.
Every failure raises :class:`StError`; nothing falls back to the CPU.
"""
import ctypes
import os

import numpy as np

from . import _lib
from .params import StParams, default_params
from .visual import visual_path


class StError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


def _addr(a, nelem):
    """Raw address of a contiguous float64 array with nelem elements."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError("arrays must be C-contiguous float64")
        if a.size != nelem:
            raise ValueError(f"array has {a.size} elements, expected {nelem}")
        return a.ctypes.data
    # torch tensor
    if getattr(a, "dtype", None) is None or str(a.dtype) != "torch.float64":
        raise TypeError("tensors must be float64")
    if not a.is_contiguous():
        raise TypeError("tensors must be contiguous")
    if a.numel() != nelem:
        raise ValueError(f"tensor has {a.numel()} elements, expected {nelem}")
    return a.data_ptr()


class Solver:
    """One solver context: device mirrors of the reference COMMON blocks."""

    def __init__(self, params=None, **kw):
        self.lib = _lib.load()
        self.params = params if params is not None else default_params(**kw)
        p = self.params
        self.shape = (p.nx, p.nz, p.ny)
        self.n3 = p.nx * p.ny * p.nz
        h = ctypes.c_void_p()
        st = self.lib.st_create(ctypes.byref(p), ctypes.byref(h))
        if st != 0:
            raise StError(st, "st_create failed: " + self.lib.st_status_string(st).decode())
        self._h = h

    # -- plumbing ---------------------------------------------------------
    def _check(self, st, what):
        if st != 0:
            msg = self.lib.st_last_error(self._h).decode(errors="replace")
            raise StError(st, f"{what}: {msg}")

    def _a(self, a, nf=1):
        return _addr(a, nf * self.n3)

    def _y(self, Y):
        """Mass-fraction argument: None (NULL) is allowed in the periodic family."""
        return None if Y is None else self._a(Y)

    def close(self):
        if getattr(self, "_h", None):
            self.lib.st_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, n=None):
        return np.zeros(self.shape if n is None else (n,) + self.shape)

    # -- state and COMMON blocks -----------------------------------------
    def set_state(self, Q, Y=None):
        self._check(self.lib.st_set_state(self._h, self._a(Q, 5), self._y(Y)), "st_set_state")

    def get_state(self, Q=None, Y=None):
        Q = self.field(5) if Q is None else Q
        Y = self.field() if Y is None else Y
        self._check(self.lib.st_get_state(self._h, self._a(Q, 5), self._a(Y)), "st_get_state")
        return Q, Y

    def set_tstep(self, t):
        self._check(self.lib.st_set_tstep(self._h, float(t)), "st_set_tstep")

    def get_tstep(self):
        t = ctypes.c_double()
        self._check(self.lib.st_get_tstep(self._h, ctypes.byref(t)), "st_get_tstep")
        return t.value

    def get_common(self, name, out=None):
        nf = 5 if name in ("dQ", "QW") else 1
        out = self.field(nf if nf > 1 else None) if out is None else out
        self._check(self.lib.st_get_common(self._h, name.encode(), self._a(out, nf)), "st_get_common")
        return out

    def set_common(self, name, arr):
        nf = 5 if name in ("dQ", "QW") else 1
        self._check(self.lib.st_set_common(self._h, name.encode(), self._a(arr, nf)), "st_set_common")

    # -- line solvers (src/tridiagonal.f90, src/pentadiagonal.f90) ----------
    def tridiagonal(self, A, B, C, R, n, lot, nper=0):
        N = n * lot
        self._check(self.lib.st_tridiagonal(self._h, _addr(A, N), _addr(B, N), _addr(C, N), _addr(R, N),
                                            n, lot, nper), "tridiagonal")

    def pentadiagonal(self, A, B, C, D, E, R, n, lot, nper=0):
        N = n * lot
        self._check(self.lib.st_pentadiagonal(self._h, _addr(A, N), _addr(B, N), _addr(C, N), _addr(D, N),
                                              _addr(E, N), _addr(R, N), n, lot, nper), "pentadiagonal")

    # -- physics (reference names) -----------------------------------------
    def Compute_gamma(self, Y):
        self._check(self.lib.st_compute_gamma(self._h, self._a(Y)), "Compute_gamma")

    def RHS(self, Q, Qrhs, Y=None):
        self._check(self.lib.st_rhs(self._h, self._a(Q, 5), self._a(Qrhs, 5), self._y(Y)), "RHS")

    def Compute_hyper(self, Q, Y=None):
        self._check(self.lib.st_compute_hyper(self._h, self._a(Q, 5), self._y(Y)), "Compute_hyper")

    def Hyper_RHS(self, Q, Qrhs, Y=None):
        self._check(self.lib.st_hyper_rhs(self._h, self._a(Q, 5), self._a(Qrhs, 5), self._y(Y)), "Hyper_RHS")

    def Species_RHS(self, Q, Qrhs, Y, Yrhs):
        self._check(self.lib.st_species_rhs(self._h, self._a(Q, 5), self._a(Qrhs, 5), self._a(Y),
                                            self._a(Yrhs)), "Species_RHS")

    def bc_RHS(self, Q, Qrhs, Y, Yrhs, time=0.0):
        self._check(self.lib.st_bc_rhs(self._h, self._a(Q, 5), self._a(Qrhs, 5), self._a(Y), self._a(Yrhs),
                                       float(time)), "bc_RHS")

    def Sponge_Forcing(self, Q, Qrhs, Y, Yrhs):
        self._check(self.lib.st_sponge_forcing(self._h, self._a(Q, 5), self._a(Qrhs, 5), self._a(Y),
                                               self._a(Yrhs)), "Sponge_Forcing")

    def Fix_Pressure(self, Q, Y=None):
        self._check(self.lib.st_fix_pressure(self._h, self._a(Q, 5), self._y(Y)), "Fix_Pressure")

    def Compact_Filter(self, F, F0, N):
        self._check(self.lib.st_compact_filter(self._h, self._a(F, N), self._a(F0, N), N), "Compact_Filter")

    def Gaussian_Filter(self, F, Fg, N):
        self._check(self.lib.st_gaussian_filter(self._h, self._a(F, N), self._a(Fg, N), N), "Gaussian_Filter")

    def Compute_CFL(self, Q):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.st_compute_cfl(self._h, self._a(Q, 5), ctypes.byref(a), ctypes.byref(b)),
                    "Compute_CFL")
        return a.value, b.value

    def Compute_Tstep(self, Q, Y, cfl_resv, step):
        t = ctypes.c_double()
        self._check(self.lib.st_compute_tstep(self._h, self._a(Q, 5), self._y(Y), float(cfl_resv), int(step),
                                              ctypes.byref(t)), "Compute_Tstep")
        return t.value

    def LDDRK4(self, time, step):
        """LDDRK4(time, step) on the resident state; returns (time, step)."""
        t, s = ctypes.c_double(time), ctypes.c_int(step)
        self._check(self.lib.st_lddrk4(self._h, ctypes.byref(t), ctypes.byref(s)), "LDDRK4")
        return t.value, s.value

    def step(self, time, step):
        """Compute_CFL + Compute_Tstep + LDDRK4 (src/main_mf.f:137-143)."""
        t, s = ctypes.c_double(time), ctypes.c_int(step)
        self._check(self.lib.st_step(self._h, ctypes.byref(t), ctypes.byref(s)), "step")
        return t.value, s.value

    def step_async(self, step):
        """Enqueue one main-loop step without waiting (graph replay from step 2)."""
        self._check(self.lib.st_step_async(self._h, int(step)), "st_step_async")

    def get_time(self):
        t = ctypes.c_double()
        self._check(self.lib.st_get_time(self._h, ctypes.byref(t)), "st_get_time")
        return t.value

    def set_time(self, t):
        self._check(self.lib.st_set_time(self._h, float(t)), "st_set_time")

    def done(self):
        """True when every operation enqueued on the context has finished."""
        st = self.lib.st_query(self._h)
        if st < 0:
            self._check(st, "st_query")
        return st == 1

    # -- Output-side diagnostics (src/out_mf.f:671-705) ---------------------
    def Compute_Grad(self, Grad=None):
        """Compute_Grad (src/grad_sym.f:13): returns (Grad, MaxDil, Enstrophy),
        Grad = (w_x, w_y, w_z, dilatation) of the context's state."""
        Grad = self.field(4) if Grad is None else Grad
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.st_compute_grad(self._h, self._a(Grad, 4), ctypes.byref(a), ctypes.byref(b)),
                    "Compute_Grad")
        return Grad, a.value, b.value

    def Compute_SRM_Stats(self):
        """Compute_SRM_Stats (pproc/pproc_mf.f:4): returns (hmix, tke_total,
        shell-averaged radial velocity, shell-averaged Y)."""
        na = ctypes.c_int()
        self._check(self.lib.st_shell_count(self._h, ctypes.byref(na)), "st_shell_count")
        ur, ya = np.zeros(na.value), np.zeros(na.value)
        h, t = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.st_compute_srm_stats(self._h, ctypes.byref(h), ctypes.byref(t),
                                                  ur.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                  ya.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                    "Compute_SRM_Stats")
        return h.value, t.value, ur, ya

    def Generate_Shock_Surface(self):
        """Generate_Shock_Surface (src/shock.f:163): returns (rad_avg, rad_skew_rms)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.st_generate_shock_surface(self._h, ctypes.byref(a), ctypes.byref(b)),
                    "Generate_Shock_Surface")
        return a.value, b.value

    def MakePaddedArrays(self, Grad=None):
        """MakePaddedArrays (src/vis_silo_mf.f:440): returns (W, xx, yy, zz),
        W (11, Mx+1, Mz+1, My+1) = u, v, w, rho, P, w_x, w_y, w_z,
        dilatation, gamma_eff, Y at the nodes of the grid padded by one node
        per direction.  Grad: the 4 fields of Compute_Grad, or None to
        compute them first."""
        nx, nz, ny = self.shape
        W = np.zeros((11, nx + 1, nz + 1, ny + 1))
        xx, yy, zz = np.zeros(nx + 1), np.zeros(ny + 1), np.zeros(nz + 1)
        g = None if Grad is None else self._a(Grad, 4)
        self._check(self.lib.st_make_padded_arrays(self._h, g, W.ctypes.data, xx.ctypes.data, yy.ctypes.data,
                                                   zz.ctypes.data), "MakePaddedArrays")
        return W, xx, yy, zz

    def Write_Visual_Silo(self, time, step, vis_path, prefix, cue_vis, Grad=None):
        """Write_Visual_Silo (src/vis_silo_mf.f:7): the visual fields as one
        legacy VTK rectilinear-grid file (the Silo library is not part of
        this build); returns its path, <vis_path>/<ddd>/<prefix>.000.vtk."""
        g = None if Grad is None else self._a(Grad, 4)
        self._check(self.lib.st_write_visual(self._h, g, os.fsencode(vis_path), os.fsencode(prefix), int(cue_vis),
                                             float(time), int(step)), "Write_Visual_Silo")
        return visual_path(vis_path, prefix, cue_vis)

    def monitors(self):
        out = np.zeros(10)
        self._check(self.lib.st_get_monitors(self._h, out.ctypes.data), "st_get_monitors")
        return out

    def sync(self):
        self._check(self.lib.st_sync(self._h), "st_sync")


def _make_line_op(cname, kind):
    if kind == "d1":
        def op(self, F, dF, iadd, cadd):
            self._check(getattr(self.lib, cname)(self._h, self._a(F), self._a(dF), int(iadd), float(cadd)), cname)
    elif kind == "d2":
        def op(self, F, dF, d2F, iadd):
            dptr = self._a(dF) if (iadd or dF is not None) else None
            self._check(getattr(self.lib, cname)(self._h, self._a(F), dptr, self._a(d2F), int(iadd)), cname)
    else:
        def op(self, F, F0):
            self._check(getattr(self.lib, cname)(self._h, self._a(F), self._a(F0)), cname)
    op.__name__ = cname
    return op


for _d in ("X", "Y", "Z"):
    for _s in ("sym", "asym"):
        setattr(Solver, f"DFD{_d}_{_s}", _make_line_op(f"st_dfd{_d.lower()}_{_s}", "d1"))
        setattr(Solver, f"D2FD{_d}2_{_s}", _make_line_op(f"st_d2fd{_d.lower()}2_{_s}", "d2"))
        setattr(Solver, f"Compact_Filter_{_d}_{_s}", _make_line_op(f"st_compact_filter_{_d.lower()}_{_s}", "f"))
    setattr(Solver, f"Gaussian_Filter_{_d}", _make_line_op(f"st_gaussian_filter_{_d.lower()}", "f"))
    # periodic family (src/derivCDopt6_periodic.f, src/filters_periodic.f)
    setattr(Solver, f"DFD{_d}", _make_line_op(f"st_dfd{_d.lower()}", "d1"))
    setattr(Solver, f"D2FD{_d}2", _make_line_op(f"st_d2fd{_d.lower()}2", "d2"))
    setattr(Solver, f"Compact_Filter_{_d}", _make_line_op(f"st_compact_filter_{_d.lower()}", "f"))

__all__ = ["Solver", "StError", "StParams", "default_params"]


class Batch:
    """A batch context: ``ncase`` independent cases of one grid size and one
    parameter set, stepped together (one launch per operator for all active
    cases; each case keeps its own time step, time and step count).  Cases
    0 .. active-1 are stepped."""

    def __init__(self, params, ncase):
        self.lib = _lib.load()
        self.params = params
        p = params
        self.shape = (p.nx, p.nz, p.ny)
        self.n3 = p.nx * p.ny * p.nz
        self.ncase = int(ncase)
        h = ctypes.c_void_p()
        st = self.lib.st_create_batch(ctypes.byref(p), self.ncase, ctypes.byref(h))
        if st != 0:
            raise StError(st, "st_create_batch failed: " + self.lib.st_status_string(st).decode())
        self._h = h
        self.active = self.ncase

    def _check(self, st, what):
        if st != 0:
            msg = self.lib.st_last_error(self._h).decode(errors="replace")
            raise StError(st, f"{what}: {msg}")

    def close(self):
        if getattr(self, "_h", None):
            self.lib.st_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_active(self, n):
        self._check(self.lib.st_set_active(self._h, int(n)), "st_set_active")
        self.active = int(n)

    def start(self, k, Q, Y=None, time=0.0):
        """Case k's state, time and step count 0, and its set-up before the
        main loop (Compute_gamma, Compute_hyper)."""
        self._check(self.lib.st_case_start(self._h, int(k), _addr(Q, 5 * self.n3),
                                           None if Y is None else _addr(Y, self.n3), float(time)),
                    "st_case_start")

    def get(self, k, Q=None, Y=None):
        """(Q, Y, time, step) of case k."""
        Q = np.zeros((5,) + self.shape) if Q is None else Q
        Y = np.zeros(self.shape) if Y is None else Y
        t = ctypes.c_double()
        n = ctypes.c_int()
        self._check(self.lib.st_case_get(self._h, int(k), _addr(Q, 5 * self.n3), _addr(Y, self.n3),
                                         ctypes.byref(t), ctypes.byref(n)), "st_case_get")
        return Q, Y, t.value, n.value

    def move(self, src, dst):
        self._check(self.lib.st_case_move(self._h, int(src), int(dst)), "st_case_move")

    def step_async(self):
        self._check(self.lib.st_batch_step_async(self._h), "st_batch_step_async")

    def done(self):
        r = self.lib.st_query(self._h)
        if r < 0:
            self._check(r, "st_query")
        return r == 1

    def sync(self):
        self._check(self.lib.st_sync(self._h), "st_sync")

    def memory_bytes(self):
        b = ctypes.c_longlong()
        self._check(self.lib.st_memory(self._h, ctypes.byref(b)), "st_memory")
        return b.value

    def launch_count(self):
        c = ctypes.c_longlong()
        self._check(self.lib.st_launch_count(self._h, ctypes.byref(c)), "st_launch_count")
        return c.value

