"""GPU parity of the Euler residual and RK stepping against the FP64 oracle.

Tolerances (FP64 path, from the project specification): relative L2 <= 1e-12 per
residual / RK stage, <= 1e-10 after 100 steps.  FP32-bulk path: relative L2
density error <= 1e-5 per residual.
"""
import numpy as np
import pytest

from oracle import oracle as O
import horses2d_b200 as hg
from cases_util import vortex_case, perturbed, rel_l2, load_mesh, dirichlet_state

pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-12
TOL_100 = 1e-10


def gpu_from(orc, params, precision=hg.PREC_FP64):
    return hg.GpuDGSEM(orc.export_mesh(), mach=params["mach"], node_type=params["node_type"],
                       riemann=params["riemann"], bcs=params["bcs"], precision=precision)


@pytest.mark.parametrize("nodes,N,riemann", [(O.LGL, 4, O.ROE), (O.LG, 4, O.ROE), (O.LGL, 3, O.HLL),
                                             (O.LG, 5, O.LXF), (O.LGL, 7, O.ROE), (O.LG, 2, O.HLL)])
def test_residual_periodic_vortex(nodes, N, riemann):
    orc, Q0, prm = vortex_case(n=8, N=N, nodes=nodes, riemann=riemann)
    Q = perturbed(Q0, 0.02, seed=N)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = gpu_from(orc, prm)
    g.set_state(Q)
    out = g.compute_time_derivative(0.0)
    assert rel_l2(out, ref) <= TOL_STAGE
    res = g.residuals()
    assert np.allclose(res, np.abs(ref.reshape(-1, 4)).max(0), rtol=1e-11)


@pytest.mark.parametrize("case", ["vortex", "supersonic_jumps"])
def test_exact_riemann_solver(case):
    """Exact Riemann solver (Newton on the star pressure, its own face-flux kernel): subsonic vortex
    faces, and a Mach 1.5 stream with density / pressure jumps that reaches the supersonic, shock and
    fan branches; residual and 10 RK3 steps."""
    from horses2d_b200 import mesh as hmesh, cases as hcases
    mach = 0.5 if case == "vortex" else 1.5
    m = hmesh.cartesian(8, 8, -5.0, 5.0, -5.0, 5.0)
    orc = O.Oracle(m, 4, nodes=O.LG, riemann=O.EXACT, mach=mach, bcs=hmesh.periodic_bcs_cartesian())
    X = orc.coords()
    if case == "vortex":
        Q = perturbed(hcases.isentropic_vortex(X[:, 0], X[:, 1], mach=mach).ravel(), 0.02, seed=21)
    else:
        left = X[:, 0] < 0.3
        rho = np.where(left, 1.0, 0.3)
        p = np.where(left, 1.0, 0.25) * (1.0 + 0.5 * (X[:, 1] > 1.1))
        u = np.where(left, 1.0, -0.4) + 0.3 * np.sin(X[:, 1])
        v = 0.4 * np.cos(X[:, 0])
        Q = perturbed(np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], 1).ravel(),
                      0.01, seed=22)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = hg.GpuDGSEM(orc.export_mesh(), mach=mach, node_type=hg.NODES_LG, riemann=hg.EXACT,
                    bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    g.set_state(Q)
    g.profile(True)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= TOL_STAGE
    assert g.kernel_times()["face_flux"][1] == 1      # one exact-flux launch ahead of the stage kernel
    g.profile(False)
    dt = orc.estimate_dt(0.1, 1.0)
    for s in range(10):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 10, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STAGE * 10


def test_rk3_stage_and_100_steps():
    orc, Q0, prm = vortex_case(n=16, N=4)
    orc.set_state(Q0)
    g = gpu_from(orc, prm)
    g.set_state(Q0)
    dt = orc.estimate_dt(0.4, 1.0)
    assert abs(g.estimate_time_step(0.4, 1.0) - dt) <= 1e-14 * dt
    orc.time_step(O.RK3, 0.0, dt)
    g.time_step(hg.SCHEME_RK3, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STAGE
    for s in range(1, 100):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 99, dt, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_100


@pytest.mark.parametrize("scheme", [O.EULER, O.RK5])
def test_other_schemes(scheme):
    orc, Q0, prm = vortex_case(n=8, N=5, nodes=O.LG)
    orc.set_state(Q0)
    g = gpu_from(orc, prm)
    g.set_state(Q0)
    dt = 0.5 * orc.estimate_dt(0.4, 1.0)
    for s in range(5):
        orc.time_step(scheme, s * dt, dt)
        g.time_step(scheme, s * dt, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STAGE * 10


def test_curved_mesh_walls_and_dirichlet():
    """Reference cylinder mesh (curved circle edges) at uniform order: Euler wall + free-stream Dirichlet."""
    m = load_mesh("CylinderBench")
    mach = 0.3
    bcs = [dict(type=O.BC_DIRICHLET, mach=mach)] * 4 + [dict(type=O.BC_EULERWALL)]
    orc = O.Oracle(m, 4, nodes=O.LGL, riemann=O.LXF, mach=mach, bcs=bcs)
    # curved boundary edges (kind 5) on the circle, no mortars (kinds 2, 3)
    assert orc.edge_count(5) > 0 and orc.edge_count(2) == 0 and orc.edge_count(3) == 0
    q = dirichlet_state(orc, mach)
    Q = perturbed(np.tile(q, orc.ndof // 4), 0.01, seed=7)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    gbcs = [dict(type=hg.BC_DIRICHLET, state=q)] * 4 + [dict(type=hg.BC_EULERWALL)]
    g = hg.GpuDGSEM(orc.export_mesh(), mach=mach, node_type=hg.NODES_LGL, riemann=hg.LXF, bcs=gbcs)
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= TOL_STAGE


def test_fp32_bulk_path():
    """FP32 bulk arithmetic with the FP64 state accumulator: the residual carries FP32
    rounding (relative 1e-4 bound on the derivative); the stepped density stays within
    the 1e-5 relative L2 target of the FP64 oracle."""
    orc, Q0, prm = vortex_case(n=8, N=4)
    orc.set_state(Q0)
    ref = orc.time_derivative(0.0)
    g = gpu_from(orc, prm, precision=hg.PREC_FP32)
    g.set_state(Q0)
    out = g.compute_time_derivative(0.0).reshape(-1, 4)
    assert rel_l2(out, ref.reshape(-1, 4)) <= 1e-4
    dt = orc.estimate_dt(0.4, 1.0)
    for s in range(20):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 20, 0.0, dt)
    rho_g, rho_o = g.state().reshape(-1, 4)[:, 0], orc.state().reshape(-1, 4)[:, 0]
    assert rel_l2(rho_g, rho_o) <= 1e-5


@pytest.mark.parametrize("nodes,N", [(O.LGL, 4), (O.LG, 6)])
def test_affine_path_with_package_mesh_builder(nodes, N):
    """The package's own box builder (affine kernel path) against the oracle's reference construction."""
    from horses2d_b200 import mesh as hmesh, cases
    nx, ny = 7, 5
    m = hmesh.cartesian(nx, ny, -5.0, 5.0, -4.0, 4.0)
    orc = O.Oracle(m, N, nodes=nodes, riemann=O.ROE, mach=0.5, bcs=hmesh.periodic_bcs_cartesian())
    X = orc.coords()
    Q = perturbed(cases.isentropic_vortex(X[:, 0], X[:, 1]).ravel(), 0.01, seed=3)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = hg.GpuDGSEM(hmesh.box_descriptor(nx, ny, -5.0, 5.0, -4.0, 4.0, N, nodes), mach=0.5, node_type=nodes,
                    riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    assert g.info()["affine"]
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= TOL_STAGE
    dt = orc.estimate_dt(0.4, 1.0)
    for s in range(10):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 10, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_100
