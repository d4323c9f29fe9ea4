"""Writes tests/golden/oracle_16.npz: oracle outputs on seeded inputs.

The reference ships no test vectors for this path and cannot be compiled here,
so these fixtures pin the oracle (and through it the CUDA library) against
itself across builds: any change to the oracle's arithmetic shows up as a
fixture mismatch.  Inputs are regenerated from their seeds by the tests and
checked against the stored input checksums first.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GRID = (16, 16, 16)          # nx, ny, nz
OUT = os.path.join(HERE, "oracle_16.npz")

# (kind, direction, asym) of the single-call fixtures
OPS = [("dfd", 0, 0), ("dfd", 1, 1), ("dfd", 2, 1), ("d2fd2", 2, 0), ("filter", 1, 0),
       ("filter", 0, 1), ("gauss", 0, 0)]


def case_params():
    from shock_turbulence_b200 import default_params
    return default_params(*GRID, re=100.0)


def inputs():
    """Seeded inputs: a random field F and the blast-in-turbulence state."""
    from shock_turbulence_b200.initial import blast_in_turbulence
    p = case_params()
    F = np.random.default_rng(2024).standard_normal((p.nx, p.nz, p.ny))
    Q, Y = blast_in_turbulence(p, k0=4.0, mach_t=0.2, p_ratio=20.0, radius_cells=3.0, seed=7)
    return p, F, Q, Y


def op_name(kind, d, asym):
    return f"{kind}_{'xyz'[d]}_{'asym' if asym else 'sym'}"


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def outputs(oracle_py, p, F, Q, Y):
    """Every fixture the tests compare: name -> array."""
    o = oracle_py.Oracle(p)
    out = {}
    for kind, d, asym in OPS:
        r = np.zeros_like(F)
        if kind == "dfd":
            o.dfd(d, asym, F, r, 0, 1.0)
        elif kind == "d2fd2":
            o.d2fd2(d, asym, F, np.zeros_like(F), r, 1)
        elif kind == "filter":
            o.filter(d, asym, F, r)
        else:
            o.gauss(d, F, r)
        out[op_name(kind, d, asym)] = r
    o.set_state(Q, Y)
    o.compute_gamma(Y)
    Qrhs = np.zeros_like(Q)
    o.rhs(Q, Qrhs, Y)
    out["rhs"] = Qrhs
    o.compute_hyper(Q, Y)
    t, s = 0.0, 0
    for _ in range(2):
        t, s = o.step(t, s)
    Qs, Ys = o.get_state()
    out["step2_Q"], out["step2_Y"] = Qs, Ys
    out["step2_time"] = np.array([t])
    return out


def main():
    import oracle_py
    oracle_py.build()
    p, F, Q, Y = inputs()
    out = outputs(oracle_py, p, F, Q, Y)
    np.savez_compressed(OUT, input_digest=np.array(digest(F, Q, Y)), **out)
    print(OUT, os.path.getsize(OUT), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
