"""Restart format and synthetic initial conditions (shock_turbulence_b200.initial).

- Restart files: the byte layout of Write_Restart (src/out_mf.f:469-551):
  gsizes = (Ny, Nz, Nx, 6) as int32, time as float64, step as int32, then
  Q_write(Ny,Nz,Nx,6) in Fortran order from byte 5*4 + 8 = 28 (the file view
  displacement disp = 5*intSize + realSize), native byte order; a write/read
  round trip returns the same bits.
- The turbulence generator: solenoidal to rounding in spectral space (off
  the Nyquist planes, which hold almost no energy), the
  shell spectrum E(k) peaks at k0 and follows k^4 exp(-2 (k/k0)^2), the rms
  velocity per component is M_t / sqrt(3) (u_rms when given), and the
  background is rho = 1, p = 1/gamma (sound speed 1).
- The blast deposit: peak pressure ratio at the symmetry corner, background
  pressure far from it.
"""
import struct

import numpy as np
import pytest

from shock_turbulence_b200.initial import (blast_in_turbulence, periodic_turbulence, read_restart,
                                           solenoidal_velocity, write_restart)
from shock_turbulence_b200.params import default_params, periodic_params


def test_restart_layout_and_round_trip(tmp_path):
    nx, ny, nz = 12, 8, 10
    rng = np.random.default_rng(4)
    Q = rng.standard_normal((5, nx, nz, ny))
    Y = rng.uniform(size=(nx, nz, ny))
    path = tmp_path / "case.restart.82"
    write_restart(path, Q, Y, 1.25, 37)
    raw = path.read_bytes()
    assert len(raw) == 28 + 8 * 6 * nx * ny * nz
    gs = struct.unpack("=4i", raw[:16])
    assert gs == (ny, nz, nx, 6)                      # gsizes(1..4) = Ny, Nz, Nx, 6
    assert struct.unpack("=d", raw[16:24])[0] == 1.25
    assert struct.unpack("=i", raw[24:28])[0] == 37
    body = np.frombuffer(raw, dtype=np.float64, offset=28)

    def at(j, k, i, l):                               # Q_write(J,K,I,L), 0-based, Fortran order
        return body[j + ny * (k + nz * (i + nx * l))]

    for (j, k, i, l) in [(0, 0, 0, 0), (3, 2, 5, 1), (ny - 1, nz - 1, nx - 1, 4), (1, 7, 9, 3)]:
        assert at(j, k, i, l) == Q[l, i, k, j]
    assert at(2, 3, 4, 5) == Y[4, 3, 2]
    Q2, Y2, t2, s2 = read_restart(path)
    assert t2 == 1.25 and s2 == 37
    assert np.array_equal(Q2, Q) and np.array_equal(Y2, Y)


def test_restart_rejects_other_variable_counts(tmp_path):
    path = tmp_path / "bad.restart"
    with open(path, "wb") as f:
        np.array([4, 4, 4, 5], dtype=np.int32).tofile(f)
        np.array([0.0], dtype=np.float64).tofile(f)
        np.array([0], dtype=np.int32).tofile(f)
        np.zeros(5 * 64).tofile(f)
    with pytest.raises(ValueError):
        read_restart(path)


def spectrum(u, v, w):
    """Shell-summed kinetic energy spectrum over integer |k| bins."""
    nx, nz, ny = u.shape
    kx = np.fft.fftfreq(nx) * nx
    kz = np.fft.fftfreq(nz) * nz
    ky = np.fft.fftfreq(ny) * ny
    KX, KZ, KY = np.meshgrid(kx, kz, ky, indexing="ij")
    kmag = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    e = sum(np.abs(np.fft.fftn(f)) ** 2 for f in (u, v, w)) * 0.5 / u.size ** 2
    bins = np.rint(kmag).astype(int)
    return np.bincount(bins.ravel(), weights=e.ravel())


@pytest.mark.parametrize("k0", [4.0, 8.0])
def test_turbulence_is_solenoidal_with_the_specified_spectrum(k0):
    n, urms = 64, 0.1
    u, v, w = solenoidal_velocity((n, n, n), k0, urms, seed=0)
    # rms per component
    assert abs(np.sqrt((u ** 2 + v ** 2 + w ** 2).mean() / 3.0) - urms) < 1e-14
    # spectral divergence with the generator's own wavenumbers, away from
    # the Nyquist planes (|k_i| = n/2, whose sign a real field cannot carry)
    k = np.fft.fftfreq(n) * n
    KX, KZ, KY = np.meshgrid(k, k, k, indexing="ij")
    uh, vh, wh = (np.fft.fftn(f) for f in (u, v, w))
    div = KX * uh + KY * vh + KZ * wh
    inner = (np.abs(KX) < n // 2) & (np.abs(KY) < n // 2) & (np.abs(KZ) < n // 2)
    scale = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2).max() * max(np.abs(x).max() for x in (uh, vh, wh))
    assert np.abs(div[inner]).max() <= 1e-12 * scale
    # the Nyquist planes carry almost no energy for k0 <= n/8
    e = np.abs(uh) ** 2 + np.abs(vh) ** 2 + np.abs(wh) ** 2
    assert e[~inner].sum() <= 1e-8 * e.sum()
    # shell spectrum: peak at k0, shape k^4 exp(-2 (k/k0)^2)
    E = spectrum(u, v, w)
    kk = np.arange(E.size)
    assert abs(int(np.argmax(E[1:n // 2])) + 1 - k0) <= 1
    model = kk ** 4.0 * np.exp(-2.0 * (kk / k0) ** 2)
    band = (kk >= 2) & (kk <= 2 * k0)
    ratio = E[band] / model[band]
    assert ratio.max() / ratio.min() < 3.0               # random amplitudes: same shape within a factor
    assert E[0] < 1e-20                                  # no mean flow


def test_config0_background_state():
    p = periodic_params(32)
    Q = periodic_turbulence(p, k0=4.0, mach_t=0.2, seed=0)
    g = p.gamma1
    assert np.array_equal(Q[3], np.ones_like(Q[3]))      # rho = 1
    u, v, w = Q[0] / Q[3], Q[1] / Q[3], Q[2] / Q[3]
    P = (g - 1.0) * (Q[4] - 0.5 * Q[3] * (u * u + v * v + w * w))
    assert np.abs(P - 1.0 / g).max() < 1e-14            # p = 1/gamma: sound speed 1
    assert abs(np.sqrt((u ** 2 + v ** 2 + w ** 2).mean() / 3.0) - 0.2 / np.sqrt(3.0)) < 1e-14


def test_blast_deposit():
    p = default_params(48, re=100.0)
    Q, Y = blast_in_turbulence(p, k0=8, mach_t=0.1, p_ratio=100.0, radius_cells=4, seed=1)
    g = p.gamma1                                          # Y = 1: gamma_eff = gamma1
    u, v, w = Q[0] / Q[3], Q[1] / Q[3], Q[2] / Q[3]
    P = (g - 1.0) * (Q[4] - 0.5 * Q[3] * (u * u + v * v + w * w))
    assert np.array_equal(Y, np.ones_like(Y))
    assert abs(P[0, 0, 0] * g - 100.0) < 1e-12           # peak ratio at the x = y = z = 0 corner
    assert abs(P[-1, -1, -1] * g - 1.0) < 1e-12          # background far away
    assert np.all(np.diff(P[:, 0, 0]) <= 1e-15)          # decays away from the corner
