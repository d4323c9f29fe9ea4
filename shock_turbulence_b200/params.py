"""Run-time parameters of the solver (ctypes mirror of ``st_params`` in
``include/st_b200.h``).

The reference fixes the grid at compile time (src/header:5-10) and reads the
flow parameters from ``srm.input.1`` (src/define_nonperiodic_mf.f:17-84);
here both travel in one struct.
"""
import ctypes
import math


class StParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("x_leng", ctypes.c_double), ("y_leng", ctypes.c_double), ("z_leng", ctypes.c_double),
        ("x_start", ctypes.c_double), ("y_start", ctypes.c_double), ("z_start", ctypes.c_double),
        ("re", ctypes.c_double),
        ("re1", ctypes.c_double), ("re2", ctypes.c_double), ("pr", ctypes.c_double), ("sc", ctypes.c_double),
        ("gamma1", ctypes.c_double), ("gamma2", ctypes.c_double), ("epsilon", ctypes.c_double),
        ("vis_exp", ctypes.c_double), ("bulk_ratio", ctypes.c_double), ("t_ratio", ctypes.c_double),
        ("hyper_param", ctypes.c_int),
        ("rk_mode", ctypes.c_int),
        ("cfl_cal", ctypes.c_double),
        ("c_beta_scale", ctypes.c_double),
        ("device", ctypes.c_int),
        ("family", ctypes.c_int),
        ("precision", ctypes.c_int),
    ]


FAMILY_MF = 0          # two-species symmetric octant (src/main_mf.f)
FAMILY_PERIODIC = 1    # single-fluid triply periodic box (src/main.f)
PRECISION_FP64 = 0     # every array in double (the reference's REAL*8 build)
PRECISION_FP32 = 1     # float intermediates; double state, accumulators, state filter, pressure recovery


def default_params(nx, ny=None, nz=None, length=2.0 * math.pi, **kw):
    """Reference input values (init/srm.input.1:19-34) on an n^3 grid spanning
    [0, length] in every direction.  Keyword arguments override fields."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = StParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.x_leng = p.y_leng = p.z_leng = length
    p.x_start = p.y_start = p.z_start = 0.0
    p.re = 0.0              # COMMON Re is never assigned in the reference build
    p.re1, p.re2 = 100.0, 100.0
    p.pr, p.sc = 0.7, 1.0
    p.gamma1, p.gamma2 = 1.4, 1.09
    p.epsilon = 0.198265856
    p.vis_exp = 0.76
    p.bulk_ratio = 0.0
    p.t_ratio = 1.0
    p.hyper_param = 1
    p.rk_mode = 0
    p.cfl_cal = 0.5
    p.c_beta_scale = 1.0
    p.device = 0
    p.family = FAMILY_MF
    p.precision = PRECISION_FP64
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(f"st_params has no field {k!r}")
        setattr(p, k, v)
    return p


def periodic_params(nx, ny=None, nz=None, period=2.0 * math.pi, re=100.0, gamma=1.4, **kw):
    """Single-fluid periodic box (src/define_periodic_sf.f): gamma and Re of the
    fluid, and x_leng = period*(N-1)/N as Define_Param sets it (:42)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = default_params(nx, ny, nz, family=FAMILY_PERIODIC, re=re, re1=re, gamma1=gamma)
    p.x_leng = period * (nx - 1) / nx
    p.y_leng = period * (ny - 1) / ny
    p.z_leng = period * (nz - 1) / nz
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(f"st_params has no field {k!r}")
        setattr(p, k, v)
    return p


class StRadialParams(ctypes.Structure):
    """st_radial_params of include/st_b200.h (1-D spherical-radial family)."""
    _fields_ = [
        ("gamma", ctypes.c_double), ("cfl_cal", ctypes.c_double),
        ("hyper_param", ctypes.c_int), ("rk_mode", ctypes.c_int), ("device", ctypes.c_int),
    ]


def radial_params(gamma=1.4, cfl_cal=0.5, hyper_param=1, rk_mode=0, device=0):
    p = StRadialParams()
    p.gamma, p.cfl_cal, p.hyper_param, p.rk_mode, p.device = gamma, cfl_cal, hyper_param, rk_mode, device
    return p
