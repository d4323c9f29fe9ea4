"""The LDDRK4 coefficients (src/header:247-296) as restated in the CUDA
library and in the oracle.

Both sides restate the reference's 16-digit constants.  GPU/oracle parity
would not notice a digit copied wrongly into both, so this file checks the
committed sources directly:

- every copy of each array (the _mf and periodic LDDRK4 and the radial
  kernels in the library, the _mf and radial oracles) holds the same values;
- each loop is a fourth-order 2N-storage scheme on linear problems: iterating
  W = alpha_k W + z y, y = y + beta_k W on y' = y from y = 1 gives an
  amplification polynomial equal to exp(z) through z^4 (the z^5 term is the
  low-dissipation design's own, 1/200 for the 5-stage loop);
- the oracle's stage times c1 are the abscissae those coefficients imply
  (w_k = alpha_k w_(k-1) + 1, c_(k+1) = c_k + beta_k w_k)."""
import math
import os
import re

import numpy as np
import pytest
from numpy.polynomial import polynomial as Pn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NUM = r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?"


def arrays(relpath, name):
    """All initialisers `<name>[k] = {...}` in a source file, as float lists."""
    src = open(os.path.join(ROOT, relpath)).read()
    out = []
    for m in re.finditer(r"\b" + re.escape(name) + r"\[\d+\]\s*=\s*\{([^}]*)\}", src):
        out.append([float(v) for v in re.findall(NUM, m.group(1))])
    return out


COPIES = {
    "alpha1": [("shock_turbulence_b200/csrc/st_physics.cu", "alpha1", 2),
               ("shock_turbulence_b200/csrc/st_radial.cu", "c_alpha1", 1),
               ("oracle/st_oracle.c", "alpha1_rk", 1), ("oracle/st_oracle_radial.c", "alpha1_rk", 1)],
    "beta1": [("shock_turbulence_b200/csrc/st_physics.cu", "beta1", 2),
              ("shock_turbulence_b200/csrc/st_radial.cu", "c_beta1", 1),
              ("oracle/st_oracle.c", "beta1_rk", 1), ("oracle/st_oracle_radial.c", "beta1_rk", 1)],
    "alpha2": [("shock_turbulence_b200/csrc/st_physics.cu", "alpha2", 1),
               ("shock_turbulence_b200/csrc/st_radial.cu", "c_alpha2", 1),
               ("oracle/st_oracle.c", "alpha2_hhm", 1), ("oracle/st_oracle_radial.c", "alpha2_hhm", 1)],
    "beta2": [("shock_turbulence_b200/csrc/st_physics.cu", "beta2", 1),
              ("shock_turbulence_b200/csrc/st_radial.cu", "c_beta2", 1),
              ("oracle/st_oracle.c", "beta2_hhm", 1), ("oracle/st_oracle_radial.c", "beta2_hhm", 1)],
}


def coefficients(key):
    found = []
    for path, name, count in COPIES[key]:
        got = arrays(path, name)
        assert len(got) == count, (path, name, len(got))
        found.extend(got)
    first = found[0]
    for other in found[1:]:
        assert other == first, (key, other, first)
    return first


@pytest.mark.parametrize("key", sorted(COPIES))
def test_every_copy_is_identical(key):
    vals = coefficients(key)
    assert len(vals) == (5 if key.endswith("1") else 6)


def amplification(alpha, beta):
    y, W = np.array([1.0]), np.array([0.0])
    for a, b in zip(alpha, beta):
        W = Pn.polyadd(a * W, Pn.polymulx(y))
        y = Pn.polyadd(y, b * W)
    return y


@pytest.mark.parametrize("loop", [1, 2])
def test_fourth_order_on_linear_problems(loop):
    y = amplification(coefficients(f"alpha{loop}"), coefficients(f"beta{loop}"))
    assert len(y) == (6 if loop == 1 else 7)
    for j in range(5):
        assert abs(y[j] - 1.0 / math.factorial(j)) < 1e-14, (loop, j, y[j])
    if loop == 1:
        assert abs(y[5] - 1.0 / 200.0) < 1e-14


def test_oracle_stage_times_follow_from_the_coefficients():
    alpha, beta = coefficients("alpha1"), coefficients("beta1")
    (c1,) = arrays("oracle/st_oracle.c", "c1_rk")
    w, c = 0.0, [0.0]
    for k in range(4):
        w = alpha[k] * w + 1.0
        c.append(c[-1] + beta[k] * w)
    assert np.allclose(c1, c, rtol=0, atol=1e-15), (c1, c)
