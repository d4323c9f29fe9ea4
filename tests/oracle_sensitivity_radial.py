"""Rounding sensitivity of the batched radial blasts (oracle only, CPU).

Runs the CPU oracle's radial batch (the problems of
tests/test_gpu_radial.py, seed 5) for 10, 30, 50 and 100 steps twice, the
second time from the initial state multiplied by (1 + 1e-14 * noise), for
each RK option, and prints the largest normwise relative difference over
the fields of the problems that stay finite (the 16-point problem overflows
in the oracle itself before step 100).  This is how far two runs that
differ only in rounding drift apart, which bounds the horizon of a
GPU-vs-oracle comparison.  Not collected by pytest (about a minute):

    python tests/oracle_sensitivity_radial.py
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import numpy as np  # noqa: E402
import oracle_py  # noqa: E402
from shock_turbulence_b200.initial import radial_blast  # noqa: E402
from shock_turbulence_b200.params import radial_params  # noqa: E402

LENGTHS = np.array([16, 37, 128, 500, 1024, 1025, 2047, 4096], dtype=np.int32)


def run(p, Q, nsteps):
    o = oracle_py.Radial(p)
    Qo = Q.copy()
    hyp = np.zeros(2 * int(LENGTHS.sum()))
    to = np.zeros(len(LENGTHS))
    so = np.zeros(len(LENGTHS), dtype=np.int32)
    o.batch(LENGTHS, np.full(len(LENGTHS), 2.0), Qo, hyp, to, so, nsteps)
    return Qo


for rk in (0, 1):
    p = radial_params(rk_mode=rk)
    rng = np.random.default_rng(5)
    Q = np.concatenate([radial_blast(int(n), 2.0, float(rng.uniform(10, 1000)), rng=rng).ravel() for n in LENGTHS])
    Q2 = Q * (1.0 + 1e-14 * np.random.default_rng(1).standard_normal(Q.size))
    for nsteps in (10, 30, 50, 100):
        a, b = run(p, Q, nsteps), run(p, Q2, nsteps)
        worst, off = 0.0, 0
        for n in LENGTHS:
            blk = a[3 * off:3 * (off + n)].reshape(3, n)
            if np.isfinite(blk).all():
                other = b[3 * off:3 * (off + n)].reshape(3, n)
                worst = max(worst, max(float(np.abs(other[f] - blk[f]).max() / np.abs(blk[f]).max())
                                       for f in range(3)))
            off += n
        print(f"rk_mode {rk}, {nsteps} steps: max field difference {worst:.2e}", flush=True)
