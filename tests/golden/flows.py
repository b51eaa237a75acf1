"""Initial flow fields shared by the golden generator and the tests.

Both sides evaluate the same formulas on bit-identical solution-point
coordinates, so the start states the reference ran from and the start states
the CUDA path runs from are the same arrays.  All states are SI (the
reference's pressure floors are in Pa, core/fr_operators/kernels.py:41-44).
"""

import numpy as np

GAMMA = 1.4
RHO, P = 1.225, 101325.0


def conserved(rho, u, v, w, p):
    E = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, E], axis=-1)


def vortex_state(x, y, Lx, Ly, rc, rho_inf, p_inf, u_inf, beta=5.0):
    """Isentropic vortex (the reference's tests/validation/_isentropic_vortex.py:42-71),
    centre at the box centre, core radius rc, carried by u_inf along x."""
    a_inf = np.sqrt(GAMMA * p_inf / rho_inf)
    dx = x - 0.5 * Lx
    dy = y - 0.5 * Ly
    r2 = (dx / rc) ** 2 + (dy / rc) ** 2
    swirl = (beta * a_inf / (2 * np.pi)) * np.exp(0.5 * (1 - r2))
    theta = 1 - (GAMMA - 1) * beta**2 / (8 * GAMMA * np.pi**2) * np.exp(1 - r2)
    rho = rho_inf * theta ** (1 / (GAMMA - 1))
    p = p_inf * theta ** (GAMMA / (GAMMA - 1))
    return conserved(rho, u_inf - swirl * dy / rc, swirl * dx / rc, np.zeros_like(x), p)


def c1_vortex(xyz, L=1.0):
    """The small configuration's start state: strength 5, free-stream Mach 0.5,
    core radius 0.2 L on the unit cube.  Returns (U, u_inf)."""
    u = 0.5 * np.sqrt(GAMMA * P / RHO)
    return vortex_state(xyz[..., 0], xyz[..., 1], L, L, 0.2 * L, RHO, P, u), u


def tgv_state(x, y, z, L, u0, rho0, p0):
    """Taylor-Green vortex initial field (the reference's tests/validation/test_tgv.py:96-112)."""
    k = 2 * np.pi / L
    u = u0 * np.sin(k * x) * np.cos(k * y) * np.cos(k * z)
    v = -u0 * np.cos(k * x) * np.sin(k * y) * np.cos(k * z)
    w = np.zeros_like(u)
    p = p0 + rho0 * u0**2 / 16 * (np.cos(2 * k * x) + np.cos(2 * k * y)) * (np.cos(2 * k * z) + 2)
    rho = p / p0 * rho0
    return conserved(rho, u, v, w, p)


def c3_tgv(xyz, L=1.0):
    """The precision-stress configuration's start state: Taylor-Green at Mach 0.1.
    Returns (U, u0)."""
    u0 = 0.1 * np.sqrt(GAMMA * P / RHO)
    return tgv_state(xyz[..., 0], xyz[..., 1], xyz[..., 2], L, u0, RHO, P), u0


def channel_state(x, y, z, L, rho_inf, u_inf, p_inf, seed):
    """Freestream with a smooth, seeded multi-mode perturbation (a few percent)."""
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * np.pi, size=8)
    Lx, Ly, Lz = L
    s = lambda i, a, b, c: np.sin(2 * np.pi * (a * x / Lx + b * y / Ly + c * z / Lz) + ph[i])  # noqa: E731
    rho = rho_inf * (1 + 0.02 * s(0, 1, 1, 0) + 0.01 * s(1, 0, 2, 1))
    u = u_inf * (1 + 0.05 * s(2, 2, 0, 1)) * np.tanh(6 * z / Lz + 0.3)
    v = 0.04 * u_inf * s(3, 1, 1, 1)
    w = 0.03 * u_inf * s(4, 0, 1, 2)
    p = p_inf * (1 + 0.002 * s(5, 1, 0, 1))
    return conserved(rho, u, v, w, p)


# Cells of the floors case that carry the planted states, and what each trips.
FLOOR_CELLS = {
    "vacuum": 13,        # rho 1e-8, p 8.4e-4 Pa: AUSM rho >= 1e-6 and p >= 10 floors, p_floor
    "overspeed": 30,     # |u| >= 1.3e4 m/s at 2e7 Pa: positivity velocity clip at 1e4
    "negative_p": 21,    # p = -2000 Pa: AUSM p floor, positivity energy reset to p_floor
    "neg_rho_k": 5,      # rho*k < 0: positivity rho*k >= 0
    "tiny_rho_w": 38,    # rho*omega = 1e-12: positivity rho*omega >= 1e-8
    "negative_rho": 44,  # rho -0.5 at rest: positivity rho >= 1e-6 (and p_floor), AUSM floors
}


def plant_floor_states(U):
    """Overwrite the cells of FLOOR_CELLS (every solution point) with states
    far beyond the reference's floors and clamps, so that rounding cannot
    decide a branch.  U is (N, S, 7) with SST columns rho*k, rho*omega.

    Every planted state keeps a moderate temperature (about 300 K, or a few
    per cent variation) and a kinetic energy at most a few times the internal
    energy, so that its temperature and pressure are not differences of huge
    equal numbers: the viscous heat flux would otherwise depend on the
    summation order at a level far above the 1e-12 parity bar."""
    U = U.copy()
    c = FLOOR_CELLS
    rho = 1e-8
    U[c["vacuum"], :, :5] = conserved(np.full(U.shape[1], rho), 0.0, 0.0, 0.0, rho * 287.0 * 293.0)
    U[c["vacuum"], :, 5] = rho * 1e-3
    U[c["vacuum"], :, 6] = rho * 10.0
    # the cell's own (varying) velocity scaled up: a uniform velocity would
    # leave its gradient, and so the viscous work term, at rounding level
    r = U[c["overspeed"], :, 0]
    vel = U[c["overspeed"], :, 1:4] / r[:, None]
    vel = vel * (1.3e4 / np.min(np.linalg.norm(vel, axis=1)))
    U[c["overspeed"], :, :5] = conserved(r, vel[:, 0], vel[:, 1], vel[:, 2], np.full_like(r, 2.0e7))
    r = U[c["negative_p"], :, 0]
    u = U[c["negative_p"], :, 1] / r
    U[c["negative_p"], :, :5] = conserved(r, u, 0.0, 0.0, np.full_like(r, -2000.0))
    U[c["neg_rho_k"], :, 5] = -0.05 * U[c["neg_rho_k"], :, 0]
    U[c["tiny_rho_w"], :, 6] = 1e-12
    # negative density at rest; the energy makes the temperature of the
    # recovered primitive state (rho floored to 1e-10) about 293 K, so the
    # cell's temperature gradient is not a difference of huge equal numbers
    # (which would make the viscous heat flux depend on summation order)
    U[c["negative_rho"], :, :5] = 0.0
    U[c["negative_rho"], :, 0] = -0.5
    U[c["negative_rho"], :, 4] = 293.0 * 287.0 * 1e-10 / (GAMMA - 1.0)
    return U
