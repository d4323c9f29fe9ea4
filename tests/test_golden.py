"""Golden fixtures (tests/golden/oracle_16.npz, made by make_golden.py): the
oracle must reproduce them exactly, and the CUDA library must match them within
the per-call (1e-12), RHS (1e-11) and two-step (1e-10) tolerances."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, rel_err

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden  # noqa: E402

FIX = os.path.join(ROOT, "tests", "golden", "oracle_16.npz")


@pytest.fixture(scope="module")
def golden():
    g = np.load(FIX)
    p, F, Q, Y = make_golden.inputs()
    assert str(g["input_digest"]) == make_golden.digest(F, Q, Y), "seeded inputs changed"
    return g, p, F, Q, Y


def test_oracle_reproduces_fixtures(golden, oracle_mod):
    g, p, F, Q, Y = golden
    out = make_golden.outputs(oracle_mod, p, F, Q, Y)
    for name, arr in out.items():
        assert rel_err(arr, g[name]) <= 1e-14, name


@pytest.mark.gpu
def test_cuda_library_matches_fixtures(golden):
    g, p, F, Q, Y = golden
    from shock_turbulence_b200 import Solver
    s = Solver(p)
    for kind, d, asym in make_golden.OPS:
        D, par = "XYZ"[d], "asym" if asym else "sym"
        r = np.zeros_like(F)
        if kind == "dfd":
            getattr(s, f"DFD{D}_{par}")(F, r, 0, 1.0)
        elif kind == "d2fd2":
            getattr(s, f"D2FD{D}2_{par}")(F, np.zeros_like(F), r, 1)
        elif kind == "filter":
            getattr(s, f"Compact_Filter_{D}_{par}")(F, r)
        else:
            getattr(s, f"Gaussian_Filter_{D}")(F, r)
        assert rel_err(r, g[make_golden.op_name(kind, d, asym)]) <= 1e-12, (kind, d, asym)
    s.set_state(Q, Y)
    s.Compute_gamma(Y)
    Qrhs = np.zeros_like(Q)
    s.RHS(Q, Qrhs, Y)
    for f in range(5):
        assert rel_err(Qrhs[f], g["rhs"][f]) <= 1e-11, f
    s.Compute_hyper(Q, Y)
    t, st = 0.0, 0
    for _ in range(2):
        t, st = s.step(t, st)
    Qs, Ys = s.get_state()
    for f in range(5):
        assert rel_err(Qs[f], g["step2_Q"][f]) <= 1e-10, f
    assert rel_err(Ys, g["step2_Y"]) <= 1e-10
    assert abs(t - float(g["step2_time"][0])) <= 1e-12 * abs(t)
