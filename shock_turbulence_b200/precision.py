"""Error of an FP32-mode run against an FP64 run of the same case.

The FP32 mode (``precision=PRECISION_FP32``) stores the derivative, filter,
artificial-viscosity and right-hand-side intermediates in float and keeps the
state, the LDDRK4 accumulators, the compact filter of the state and the
pressure recovery in double.  Its error is stated per conserved field as
relative L2 and Linf norms of the difference."""
import numpy as np

FIELDS = ("rho_u", "rho_v", "rho_w", "rho", "rho_E")


def field_errors(Q, Qref, Y=None, Yref=None):
    """{field: (relative L2, relative Linf)} of Q against Qref, per conserved
    field (and the mass fraction when both Y are given).  L2 is
    ||Q - Qref||_2 / ||Qref||_2, Linf is max|Q - Qref| / max|Qref|."""
    out = {}
    pairs = [(FIELDS[l], Q[l], Qref[l]) for l in range(5)]
    if Y is not None and Yref is not None:
        pairs.append(("Y", Y, Yref))
    for name, a, b in pairs:
        a = np.asarray(a, dtype=np.float64).ravel()
        b = np.asarray(b, dtype=np.float64).ravel()
        d = a - b
        l2 = float(np.sqrt(np.dot(d, d)) / max(np.sqrt(np.dot(b, b)), 1e-300))
        linf = float(np.abs(d).max() / max(np.abs(b).max(), 1e-300))
        out[name] = (l2, linf)
    return out


def worst(errors):
    """Largest relative L2 and Linf over the fields."""
    return max(e[0] for e in errors.values()), max(e[1] for e in errors.values())
