"""Initial states of the benchmark workloads, in the reference's dimensionless variables.

The reference stores Q = (rho/rho_ref, rho u/(rho_ref a_ref), rho v/(rho_ref a_ref),
rho e/p_ref) with a_ref = sqrt(p_ref/rho_ref) (Physics/VariableConversion.f90:32-42,
_DIMENSIONLESS_TAU).  In those units a free stream at rest state (rho, p) = (1, 1)
has speed sqrt(gamma) M, and the total energy is p/(gamma-1) + rho|u|^2/2.
"""
import numpy as np


def isentropic_vortex(x, y, *, mach=0.5, angle_deg=45.0, beta=5.0, xc=0.0, yc=0.0, gamma=1.4):
    """Shu's isentropic vortex on a uniform stream (rho = p = 1), nodes given as flat arrays.

    Returns Q with shape [n, 4] in the reference's dimensionless variables.
    """
    th = np.deg2rad(angle_deg)
    u0 = np.sqrt(gamma) * mach * np.cos(th)
    v0 = np.sqrt(gamma) * mach * np.sin(th)
    dx, dy = x - xc, y - yc
    r2 = dx * dx + dy * dy
    f = beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
    u = u0 - f * dy
    v = v0 + f * dx
    T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * np.pi * np.pi) * np.exp(1.0 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho * T
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)], 1)


def uniform_state(n, *, mach, angle_deg=0.0, gamma=1.4):
    th = np.deg2rad(angle_deg)
    u = np.sqrt(gamma) * mach * np.cos(th)
    v = np.sqrt(gamma) * mach * np.sin(th)
    q = np.array([1.0, u, v, 1.0 / (gamma - 1.0) + 0.5 * (u * u + v * v)])
    return np.tile(q, (n, 1))


def kelvin_helmholtz(x, y, *, mach=0.3, delta=0.01, eps=1e-2, n_modes=4, seed=0, drho=0.0, gamma=1.4):
    """Doubly periodic shear layer on [0,1]^2 (p = 1): u = U tanh((y - 1/4)/delta) below y = 1/2 and
    U tanh((3/4 - y)/delta) above, U = sqrt(gamma) M, so that both layers are periodic; the transverse
    velocity carries a seeded multi-mode perturbation eps U sum_m a_m sin(2 pi m x + phi_m), damped away
    from the layers by exp(-(d/(4 delta))^2).  Density 1, or with drho > 0 a stream of density 1 + drho
    between the layers (same tanh profile).  Returns Q [n, 4] in the reference's dimensionless variables.
    """
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.5, 1.0, n_modes)
    amp /= amp.sum()
    phase = rng.uniform(0.0, 2.0 * np.pi, n_modes)
    U = np.sqrt(gamma) * mach
    u = np.where(y < 0.5, U * np.tanh((y - 0.25) / delta), U * np.tanh((0.75 - y) / delta))
    d = np.minimum(np.abs(y - 0.25), np.abs(y - 0.75))
    pert = np.zeros_like(x)
    for m in range(n_modes):
        pert += amp[m] * np.sin(2.0 * np.pi * (m + 1) * x + phase[m])
    v = eps * U * pert * np.exp(-(d / (4.0 * delta)) ** 2)
    rho = 1.0 + 0.5 * drho * (1.0 - np.where(y < 0.5, np.tanh((y - 0.25) / delta), np.tanh((0.75 - y) / delta)))
    p = np.ones_like(x)
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)], 1)


def kelvin_helmholtz_factors(n, N, xi, *, mach=0.3, delta=0.01, eps=1e-2, n_modes=4, seed=0, drho=0.0, gamma=1.4):
    """Separable factors of ``kelvin_helmholtz`` on the nodes of ``mesh.box_descriptor(n, n, 0, 1, 0, 1,
    N, ...)`` (nodes ``xi`` on [0,1]): density, streamwise velocity and the perturbation's damping as
    functions of y, the perturbation's transverse velocity (times eps U) as a function of x, each as
    [element index along the axis][node index] (rho_y, u_y, damp_y, vx_x)."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.5, 1.0, n_modes)
    amp /= amp.sum()
    phase = rng.uniform(0.0, 2.0 * np.pi, n_modes)
    U = np.sqrt(gamma) * mach
    h = 1.0 / n
    xi = np.asarray(xi, float)
    assert xi.size == N + 1
    c = (0.0 + np.arange(n) * h)[:, None] + h * xi[None, :]
    y, x = c, c
    u = np.where(y < 0.5, U * np.tanh((y - 0.25) / delta), U * np.tanh((0.75 - y) / delta))
    d = np.minimum(np.abs(y - 0.25), np.abs(y - 0.75))
    pert = np.zeros_like(x)
    for m in range(n_modes):
        pert += amp[m] * np.sin(2.0 * np.pi * (m + 1) * x + phase[m])
    vx = eps * U * pert
    damp = np.exp(-(d / (4.0 * delta)) ** 2)
    rho_y = 1.0 + 0.5 * drho * (1.0 - np.where(y < 0.5, np.tanh((y - 0.25) / delta), np.tanh((0.75 - y) / delta)))
    return rho_y, u, damp, vx


def kelvin_helmholtz_box(n, N, xi, gamma=1.4, **kw):
    """``kelvin_helmholtz`` at the nodes of ``mesh.box_descriptor(n, n, 0, 1, 0, 1, N, ...)`` as Q
    [n*n*(N+1)^2*4] in Storage%Q order (element j*n+i, node b*(N+1)+a), from the separable factors:
    equal to ``kelvin_helmholtz`` at those nodes, value for value."""
    rho_y, u, damp, vx = kelvin_helmholtz_factors(n, N, xi, gamma=gamma, **kw)
    P = N + 1
    Q = np.empty((n, n, P, P, 4))                                        # [j][i][b][a][v]
    rho = np.broadcast_to(rho_y[:, None, :, None], (n, n, P, P))
    uu = np.broadcast_to(u[:, None, :, None], (n, n, P, P))
    v = vx[None, :, None, :] * damp[:, None, :, None]
    Q[..., 0] = rho
    Q[..., 1] = rho * uu
    Q[..., 2] = rho * v
    Q[..., 3] = 1.0 / (gamma - 1.0) + 0.5 * rho * (uu * uu + v * v)
    return Q.reshape(-1)
