"""Shared set-up for the parity tests: oracle-built meshes handed to the GPU library.

The oracle (tests' checker) constructs each mesh exactly as the reference does
(QuadMesh_t after constructFromFile + ConstructZones); its flattened export is
what the Fortran shim would pass to hg_create.  Both sides then run on the same
state and their residuals / steps are compared.
"""
import os

import numpy as np

from oracle import oracle as O
from horses2d_b200 import cases, mesh as hmesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_mesh(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.mesh.npz")))


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def vortex_case(n=16, N=4, nodes=O.LGL, riemann=O.ROE, mach=0.5):
    """Periodic [-5,5]^2 isentropic vortex (beta 5, M 0.5 at 45 deg)."""
    m = hmesh.cartesian(n, n, -5.0, 5.0, -5.0, 5.0)
    orc = O.Oracle(m, N, nodes=nodes, riemann=riemann, mach=mach, bcs=hmesh.periodic_bcs_cartesian())
    X = orc.coords()
    Q0 = cases.isentropic_vortex(X[:, 0], X[:, 1], mach=mach).ravel()
    return orc, Q0, dict(mach=mach, node_type=nodes, riemann=riemann,
                         bcs=[dict(type=b["type"]) for b in hmesh.periodic_bcs_cartesian()])


def perturbed(Q0, amp, seed):
    rng = np.random.default_rng(seed)
    Q = Q0.reshape(-1, 4).copy()
    Q *= 1.0 + amp * rng.standard_normal(Q.shape)
    return Q.ravel()


def dirichlet_state(orc, mach, aoa_deg=0.0):
    """Dimensionless free-stream state of a Dirichlet zone (DirichletBC_Construct)."""
    r = orc.ref
    gamma, R = 1.4, 287.15
    T, p = r["T"], r["p"]
    V = mach * np.sqrt(gamma * R * T)
    rho = p / (R * T)
    th = np.deg2rad(aoa_deg)
    q = np.array([rho, rho * V * np.cos(th), rho * V * np.sin(th), 2.5 * p + 0.5 * rho * V * V])
    return q / np.array([r["rho"], r["rho"] * r["a"], r["rho"] * r["a"], r["p"]])
