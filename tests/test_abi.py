"""C ABI checks that need no GPU: the CUDA library loads and exports every
entry point that include/st_b200.h declares, and the ctypes binding covers
them all."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "st_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(st_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from shock_turbulence_b200 import build, _lib
    build.build()
    return _lib.load()


def test_header_declares_reference_routines():
    names = declared_functions()
    for must in ("st_dfdx_sym", "st_d2fdz2_asym", "st_compact_filter", "st_gaussian_filter_y",
                 "st_tridiagonal", "st_pentadiagonal", "st_rhs", "st_hyper_rhs", "st_species_rhs",
                 "st_bc_rhs", "st_sponge_forcing", "st_fix_pressure", "st_lddrk4", "st_compute_cfl",
                 "st_compute_tstep", "st_compute_hyper", "st_compute_gamma"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), f"libst_b200.so does not export {name}"


def test_binding_covers_header():
    from shock_turbulence_b200 import _lib
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_no_device_is_reported_not_crashed(lib):
    """Without a GPU the context constructor returns a status, never aborts."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from shock_turbulence_b200.params import default_params
    h = ctypes.c_void_p()
    st = lib.st_create(ctypes.byref(default_params(32)), ctypes.byref(h))
    assert st == -6   # ST_E_NODEVICE
    assert lib.st_status_string(st) == b"no usable CUDA device"


def test_status_strings(lib):
    assert lib.st_status_string(0) == b"ok"
    assert lib.st_status_string(-4) == b"unsupported size or mode"
