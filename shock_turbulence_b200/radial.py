"""Batched 1-D spherical-radial family on the GPU (C ABI ``st_radial_*``).

Each problem is one run of the reference's radial program (src/makefile_radial:
rhsv_radial.f, derivCDopt6_radial.f, filters_nonperiodic.f, hyper_radial.f,
lddrk4_nonperiodic_sf.f) on a line of n points; a batch advances any number
of problems of different lengths together.  Arrays are packed: problem k's
state block (u_r, rho, s = P/rho^gamma) of 3*n_k values starts at
3*sum(n_j, j<k); single fields start at sum(n_j, j<k).
"""
import ctypes

import numpy as np

from . import _lib
from .api import StError, _addr
from .params import radial_params


class RadialBatch:
    def __init__(self, lengths, x_leng, params=None):
        self.lib = _lib.load()
        self.params = params if params is not None else radial_params()
        self.lengths = np.ascontiguousarray(lengths, dtype=np.int32)
        self.x_leng = np.ascontiguousarray(x_leng, dtype=np.float64)
        self.nprob = len(self.lengths)
        self.npts = int(self.lengths.sum())
        self.offsets = np.zeros(self.nprob, dtype=np.int64)
        self.offsets[1:] = np.cumsum(self.lengths)[:-1]
        h = ctypes.c_void_p()
        st = self.lib.st_radial_create(ctypes.byref(self.params), self.nprob,
                                       self.lengths.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                       self.x_leng.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       ctypes.byref(h))
        if st != 0:
            raise StError(st, "st_radial_create failed: " + self.lib.st_status_string(st).decode())
        self._h = h

    def _check(self, st, what):
        if st != 0:
            raise StError(st, f"{what}: {self.lib.st_radial_last_error(self._h).decode(errors='replace')}")

    def close(self):
        if getattr(self, "_h", None):
            self.lib.st_radial_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, nf=1):
        return np.zeros(nf * self.npts)

    # state
    def set_state(self, Q):
        self._check(self.lib.st_radial_set_state(self._h, _addr(Q, 3 * self.npts)), "st_radial_set_state")

    def get_state(self, Q=None):
        Q = self.field(3) if Q is None else Q
        self._check(self.lib.st_radial_get_state(self._h, _addr(Q, 3 * self.npts)), "st_radial_get_state")
        return Q

    def get_hyper(self):
        h = self.field(2)
        self._check(self.lib.st_radial_get_hyper(self._h, _addr(h, 2 * self.npts)), "st_radial_get_hyper")
        return h

    def get_time(self):
        t = np.zeros(self.nprob)
        s = np.zeros(self.nprob, dtype=np.int32)
        self._check(self.lib.st_radial_get_time(self._h, t.ctypes.data, s.ctypes.data), "st_radial_get_time")
        return t, s

    def step(self, nsteps=1):
        self._check(self.lib.st_radial_step(self._h, int(nsteps)), "st_radial_step")

    def step_async(self, nsteps=1):
        self._check(self.lib.st_radial_step_async(self._h, int(nsteps)), "st_radial_step_async")

    def set_stream(self, stream):
        self._check(self.lib.st_radial_set_stream(self._h, stream), "st_radial_set_stream")

    def config(self, short=None, long=None):
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.st_radial_config(self._h, ctypes.byref(a), ctypes.byref(b), 0), "st_radial_config")
        if short is not None or long is not None:
            a.value = a.value if short is None else short
            b.value = b.value if long is None else long
            self._check(self.lib.st_radial_config(self._h, ctypes.byref(a), ctypes.byref(b), 1), "st_radial_config")
        return a.value, b.value

    def tune(self):
        ms = (ctypes.c_double * 2)()
        self._check(self.lib.st_radial_tune(self._h, ms), "st_radial_tune")
        return self.config(), (ms[0], ms[1])

    def launch_count(self):
        c = ctypes.c_longlong()
        self._check(self.lib.st_radial_launch_count(self._h, ctypes.byref(c)), "st_radial_launch_count")
        return c.value

    # line operators (reference names, x direction of every problem)
    def DFDX(self, F, dF, iadd, cadd):
        self._check(self.lib.st_radial_dfdx(self._h, _addr(F, self.npts), _addr(dF, self.npts), int(iadd),
                                            float(cadd)), "DFDX")

    def D2FDX2(self, F, dF, d2F, iadd):
        self._check(self.lib.st_radial_d2fdx2(self._h, _addr(F, self.npts),
                                              _addr(dF, self.npts) if dF is not None else None,
                                              _addr(d2F, self.npts), int(iadd)), "D2FDX2")

    def Compact_Filter_X(self, F, F0):
        self._check(self.lib.st_radial_compact_filter_x(self._h, _addr(F, self.npts), _addr(F0, self.npts)),
                    "Compact_Filter_X")

    def Gaussian_Filter_X(self, F, Fg):
        self._check(self.lib.st_radial_gaussian_filter_x(self._h, _addr(F, self.npts), _addr(Fg, self.npts)),
                    "Gaussian_Filter_X")

    def RHS(self, Q, Qrhs):
        self._check(self.lib.st_radial_rhs(self._h, _addr(Q, 3 * self.npts), _addr(Qrhs, 3 * self.npts)), "RHS")

    def RHS_with_hyper(self, Q, Qrhs):
        """RHS followed by Hyper_RHS (the LDDRK4 stage order); refreshes /HYPER/."""
        self._check(self.lib.st_radial_rhs_hyper(self._h, _addr(Q, 3 * self.npts), _addr(Qrhs, 3 * self.npts)),
                    "RHS+Hyper_RHS")
