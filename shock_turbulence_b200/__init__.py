"""B200 (sm_100a) implementation of the per-stage right-hand side and LDDRK4
stage update of the compact-difference shock-turbulence solver (two-species
"_mf" family).  The compute path is ``libst_b200.so`` (CUDA, C ABI in
include/st_b200.h); this package is its host-side mirror of the reference's
subroutine interface."""
from .params import (FAMILY_MF, FAMILY_PERIODIC, PRECISION_FP32, PRECISION_FP64, StParams, default_params,  # noqa: F401
                     periodic_params)
from .api import Batch, Solver, StError  # noqa: F401
