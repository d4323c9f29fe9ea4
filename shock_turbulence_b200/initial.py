"""Synthetic initial conditions and the reference restart-file format.

The reference has no turbulence generator (its init/ programs build a
converging shock with a perturbed interface), so the seeded generator below
stands in for the benchmark inputs: a solenoidal random-phase velocity field
with spectrum E(k) ~ k^4 exp(-2 (k/k0)^2), plus an optional Gaussian pressure
deposit at the symmetry corner (the template of Add_Shock_Expanding,
src/shock.f:1-86, moved to the origin of the octant domain).

Thermodynamic background: rho = 1, p = 1/gamma (sound speed 1), so the rms
velocity per component is M_t / sqrt(3) for a turbulent Mach number M_t.

Restart files follow Write_Restart / Read_Restart (src/out_mf.f:453-662):
four int32 sizes (Ny, Nz, Nx, 6), float64 time, int32 step, then
Q(Ny,Nz,Nx,6) in Fortran order (5 conserved variables and Y), native byte
order.
"""
import numpy as np


def solenoidal_velocity(shape, k0, urms, seed):
    """Random-phase solenoidal field on a periodic grid of the given C-order
    shape (Mx, Mz, My); returns (u, v, w) with per-component rms ``urms``.
    Wavenumbers are counted in units of the box fundamental.  Every mode is
    divergence-free except those on the Nyquist planes (|k_i| = N/2), whose
    wavenumber sign a real field cannot carry; for k0 <= N/8 they hold less
    than 1e-8 of the energy."""
    rng = np.random.default_rng(seed)
    nx, nz, ny = shape
    kx = np.fft.fftfreq(nx) * nx
    kz = np.fft.fftfreq(nz) * nz
    ky = np.fft.rfftfreq(ny) * ny
    KX, KZ, KY = np.meshgrid(kx, kz, ky, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k = np.sqrt(k2)
    kk = np.where(k > 0, k, 1.0)
    spec = kk ** 4 * np.exp(-2.0 * (kk / k0) ** 2)
    amp = np.where(k > 0, np.sqrt(spec / (4.0 * np.pi * kk ** 2)), 0.0)
    comps = []
    for _ in range(3):
        ph = rng.uniform(0.0, 2.0 * np.pi, size=k.shape)
        mag = rng.normal(size=k.shape)
        comps.append(amp * mag * np.exp(1j * ph))
    # project out the component along k (divergence-free)
    dot = (comps[0] * KX + comps[1] * KY + comps[2] * KZ) / np.where(k2 > 0, k2, 1.0)
    uh = [comps[0] - dot * KX, comps[1] - dot * KY, comps[2] - dot * KZ]
    fields = [np.fft.irfftn(c, s=(nx, nz, ny), axes=(0, 1, 2)) for c in uh]
    u, v, w = fields
    rms = np.sqrt((u ** 2 + v ** 2 + w ** 2).mean() / 3.0)
    scale = urms / rms if rms > 0 else 0.0
    return u * scale, v * scale, w * scale


def blast_in_turbulence(params, k0=8.0, mach_t=0.1, p_ratio=100.0, radius_cells=4.0, seed=1,
                        y_field=None):
    """Conserved state Q (5, Mx, Mz, My) and mass fraction Y for an
    expanding blast (Gaussian energy deposit at the x=y=z=0 corner) in
    isotropic turbulence.  ``p_ratio`` <= 1 gives turbulence alone."""
    shape = (params.nx, params.nz, params.ny)
    g = params.gamma1
    urms = mach_t / np.sqrt(3.0)
    u, v, w = solenoidal_velocity(shape, k0, urms, seed)
    rho = np.ones(shape)
    p0 = 1.0 / g
    dx = params.x_leng / (params.nx - 1)
    x = params.x_start + dx * np.arange(params.nx)
    y = params.y_start + params.y_leng / (params.ny - 1) * np.arange(params.ny)
    z = params.z_start + params.z_leng / (params.nz - 1) * np.arange(params.nz)
    r2 = x[:, None, None] ** 2 + z[None, :, None] ** 2 + y[None, None, :] ** 2
    p = p0 * (1.0 + (p_ratio - 1.0) * np.exp(-r2 / (radius_cells * dx) ** 2)) if p_ratio > 1.0 \
        else np.full(shape, p0)
    Y = np.ones(shape) if y_field is None else np.asarray(y_field, dtype=np.float64)
    # gamma_eff of the mixture (Compute_gamma, src/lddrk4_nonperiodic_mf.f:342-372)
    g1, g2, eps = params.gamma1, params.gamma2, params.epsilon
    geff = ((Y * g1 / (g1 - 1.0)) + (eps * (1.0 - Y) * g2 / (g2 - 1.0))) / \
           ((Y / (g1 - 1.0)) + (eps * (1.0 - Y) / (g2 - 1.0)))
    Q = np.empty((5,) + shape)
    Q[0], Q[1], Q[2], Q[3] = rho * u, rho * v, rho * w, rho
    Q[4] = p / (geff - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.ascontiguousarray(Q), np.ascontiguousarray(Y)


def periodic_turbulence(params, k0=4.0, urms=0.1, mach_t=None, seed=0):
    """Conserved state Q (5, Mx, Mz, My) of decaying isotropic turbulence in
    the single-fluid periodic box: rho = 1, p = 1/gamma (sound speed 1), zero
    entropy fluctuation, solenoidal velocity with rms ``urms`` per component.
    When ``mach_t`` is given it sets urms = mach_t/sqrt(3) instead."""
    shape = (params.nx, params.nz, params.ny)
    if mach_t is not None:
        urms = mach_t / np.sqrt(3.0)
    u, v, w = solenoidal_velocity(shape, k0, urms, seed)
    g = params.gamma1
    rho = np.ones(shape)
    p = np.full(shape, 1.0 / g)
    Q = np.empty((5,) + shape)
    Q[0], Q[1], Q[2], Q[3] = rho * u, rho * v, rho * w, rho
    Q[4] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.ascontiguousarray(Q)


def radial_blast(n, x_leng=2.0, p_ratio=100.0, radius_cells=4.0, rho_amp=0.01, gamma=1.4, rng=None):
    """One 1-D spherical-radial blast problem on n points spanning
    -x_leng/2..x_leng/2 (r = |(i - n/2 - 1/2) DX|, src/rhsv_radial.f:55-59):
    u_r = 0, rho = 1 + rho_amp * (random-phase radial perturbation with a
    k^2 exp(-k^2/8) spectrum, max |.| = 1), P = (1/gamma) (1 + (p_ratio - 1)
    exp(-r^2 / (radius_cells DX)^2)), s = P / rho^gamma.  Returns Q (3, n)."""
    rng = np.random.default_rng(0) if rng is None else rng
    dx = x_leng / (n - 1)
    i = np.arange(1, n + 1)
    r = np.abs(((i - n // 2).astype(np.float32).astype(np.float64) - 0.5) * dx)
    R = x_leng / 2.0
    k = np.arange(1, 17)
    amp = k ** 2 * np.exp(-(k ** 2) / 8.0)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=k.size)
    pert = (amp[:, None] * np.cos(np.pi * k[:, None] * r[None, :] / R + ph[:, None])).sum(axis=0)
    pert /= np.abs(pert).max()
    rho = 1.0 + rho_amp * pert
    P = (1.0 / gamma) * (1.0 + (p_ratio - 1.0) * np.exp(-r ** 2 / (radius_cells * dx) ** 2))
    Q = np.zeros((3, n))
    Q[1] = rho
    Q[2] = P / rho ** gamma
    return Q


def radial_batch(nprob, nmin=128, nmax=4096, pmin=10.0, pmax=1000.0, seed=2, gamma=1.4, x_leng=2.0):
    """Independent radial blast problems with lengths drawn uniformly from
    [nmin, nmax] and peak pressure ratios from [pmin, pmax] (seeded).
    Returns (lengths int32, x_leng float64, packed Q): problem k's block of
    3*n_k values (u, rho, s) starts at 3*sum(n_j, j<k)."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(nmin, nmax + 1, size=nprob).astype(np.int32)
    ratios = rng.uniform(pmin, pmax, size=nprob)
    blocks = [radial_blast(int(n), x_leng, float(pr), gamma=gamma, rng=rng).ravel()
              for n, pr in zip(lengths, ratios)]
    return lengths, np.full(nprob, float(x_leng)), np.ascontiguousarray(np.concatenate(blocks))


def write_restart(path, Q, Y, time, step):
    """Write_Restart layout (src/out_mf.f:469-551)."""
    nx, nz, ny = Y.shape
    with open(path, "wb") as f:
        np.array([ny, nz, nx, 6], dtype=np.int32).tofile(f)
        np.array([time], dtype=np.float64).tofile(f)
        np.array([step], dtype=np.int32).tofile(f)
        data = np.concatenate([np.asarray(Q).reshape(5, -1), np.asarray(Y).reshape(1, -1)])
        data.astype(np.float64).tofile(f)


def read_restart(path):
    """Read_Restart layout (src/out_mf.f:563-662): returns (Q, Y, time, step)."""
    with open(path, "rb") as f:
        ny, nz, nx, nv = np.fromfile(f, dtype=np.int32, count=4)
        time = float(np.fromfile(f, dtype=np.float64, count=1)[0])
        step = int(np.fromfile(f, dtype=np.int32, count=1)[0])
        data = np.fromfile(f, dtype=np.float64, count=int(nv) * nx * ny * nz)
    if int(nv) != 6:
        raise ValueError(f"restart file holds {nv} variables, expected 6")
    data = data.reshape(6, nx, nz, ny)
    return np.ascontiguousarray(data[:5]), np.ascontiguousarray(data[5]), time, step
