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
