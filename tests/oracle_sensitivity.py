"""Rounding sensitivity of the 100-step _mf blast (oracle only, CPU).

Runs the CPU oracle twice for 100 main-loop steps on the 64^3 blast in
turbulence of tests/test_gpu_long.py, the second time from the initial state
multiplied by (1 + 1e-15 * noise), and prints the normwise relative
difference per field at a few steps.  The difference measures how far two
runs that differ only in rounding drift apart, which bounds what any
implementation that does not reproduce the reference's operation order bit
for bit can match.  Not collected by pytest (about 4 minutes on 16 cores):

    python tests/oracle_sensitivity.py [pressure ratio, default 100]
"""
import sys
import os
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
import numpy as np, oracle_py
from shock_turbulence_b200.params import default_params
from shock_turbulence_b200.initial import blast_in_turbulence
pr = float(sys.argv[1]) if len(sys.argv) > 1 else 100.0
p = default_params(64, 64, 64, re=100.0, rk_mode=0, c_beta_scale=1.75)
x = np.linspace(0, 1, p.nx)[:, None, None]
y = np.linspace(0, 1, p.ny)[None, None, :]
Yf = 0.5 + 0.5 * np.tanh(8 * (np.sqrt(x ** 2 + y ** 2) - 0.5)) * np.ones((p.nx, p.nz, p.ny))
Q, Y = blast_in_turbulence(p, k0=4, mach_t=0.1, p_ratio=pr, radius_cells=4, seed=11, y_field=Yf)
rng = np.random.default_rng(0)
Q2 = Q * (1.0 + 1e-15 * rng.standard_normal(Q.shape))
runs = []
for q in (Q, Q2):
    o = oracle_py.Oracle(p)
    o.set_state(q, Y); o.compute_gamma(Y); o.compute_hyper(q, Y)
    runs.append(o)
ts = [0.0, 0.0]; ks = [0, 0]
def rel(a, b): return float(np.abs(a - b).max() / np.abs(b).max())
for i in range(100):
    for j in range(2):
        ts[j], ks[j] = runs[j].step(ts[j], ks[j])
    if (i + 1) in (1, 10, 25, 50, 60, 70, 80, 90, 100):
        A, YA = runs[0].get_state(); B, YB = runs[1].get_state()
        e = [rel(B[l], A[l]) for l in range(5)] + [rel(YB, YA)]
        print(i + 1, "max field diff", max(e), ["%.1e" % v for v in e], flush=True)
