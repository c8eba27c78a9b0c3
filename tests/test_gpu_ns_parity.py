"""GPU parity of the Navier-Stokes residual (BR1 and interior penalty) and RK stepping against the FP64 oracle.

Cases: the reference's cylinder mesh (curved circle edges, 640 quads) with a
viscous wall, far field, Dirichlet and pressure-outlet zones; a periodic
vortex box; an O-grid built by the package's own mesh builder.
Tolerances (FP64 path): relative L2 <= 1e-12 per residual / RK stage,
<= 1e-10 after 100 steps.  FP32-bulk path: residual <= 1e-4, density after
20 RK3 steps <= 1e-5 (relative L2).
"""
import numpy as np
import pytest

from oracle import oracle as O
import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases
from cases_util import perturbed, rel_l2, load_mesh, dirichlet_state

pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-12
TOL_100 = 1e-10
MACH, RE = 0.3, 200.0


def cylinder_ns(N, nodes, viscous, ip_method=0, sigma0=1.0, wall="isothermal", riemann=O.ROE):
    """Cylinder mesh: bottom Dirichlet, top/left far field, right pressure outlet, circle viscous wall."""
    m = load_mesh("CylinderBench")
    wall_type = 1 if wall == "isothermal" else 2
    T_ref = 273.15
    obcs = [dict(type=O.BC_DIRICHLET), dict(type=O.BC_FARFIELD), dict(type=O.BC_FARFIELD),
            dict(type=O.BC_PRESSUREOUTLET, outflow_type=2),
            dict(type=O.BC_VISCOUSWALL, wall_type=wall_type, wall_T=1.1 * T_ref,
                 wall_v=(0.05, -0.02))]
    orc = O.Oracle(m, N, nodes=nodes, riemann=riemann, mach=MACH, reynolds=RE, navier_stokes=1,
                   viscous=viscous, ip_method=ip_method, sigma0_ip=sigma0, bcs=obcs)
    q = dirichlet_state(orc, MACH)
    gbcs = [dict(type=hg.BC_DIRICHLET, state=q), dict(type=hg.BC_FARFIELD, state=q),
            dict(type=hg.BC_FARFIELD, state=q), dict(type=hg.BC_PRESSUREOUTLET, state=q, outflow_type=2),
            dict(type=hg.BC_VISCOUSWALL, wall_type=wall_type, wall_T=1.1, wall_v=(0.05, -0.02))]
    kw = dict(mach=MACH, reynolds=RE, navier_stokes=1, viscous=viscous, ip_method=ip_method, sigma0_ip=sigma0,
              node_type=nodes, riemann=riemann, bcs=gbcs)
    Q0 = np.tile(q, orc.ndof // 4)
    return orc, kw, Q0


def vortex_ns(N, nodes, viscous, ip_method=0, n=8):
    m = hmesh.cartesian(n, n, -5.0, 5.0, -5.0, 5.0)
    orc = O.Oracle(m, N, nodes=nodes, riemann=O.ROE, mach=0.5, reynolds=50.0, navier_stokes=1, viscous=viscous,
                   ip_method=ip_method, sigma0_ip=2.0, bcs=hmesh.periodic_bcs_cartesian())
    X = orc.coords()
    Q0 = cases.isentropic_vortex(X[:, 0], X[:, 1], mach=0.5).ravel()
    kw = dict(mach=0.5, reynolds=50.0, navier_stokes=1, viscous=viscous, ip_method=ip_method, sigma0_ip=2.0,
              node_type=nodes, riemann=O.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    return orc, kw, Q0


def residual_pair(orc, kw, Q, precision=hg.PREC_FP64, mesh=None):
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = hg.GpuDGSEM(mesh if mesh is not None else orc.export_mesh(), precision=precision, **kw)
    g.set_state(Q)
    return g, g.compute_time_derivative(0.0), ref


@pytest.mark.parametrize("N,nodes,viscous,ip", [(4, O.LGL, O.BR1, 0), (3, O.LG, O.BR1, 0), (5, O.LG, O.IP, 0),
                                               (4, O.LGL, O.IP, 1), (2, O.LG, O.IP, 2), (6, O.LGL, O.BR1, 0)])
def test_cylinder_ns_residual(N, nodes, viscous, ip):
    orc, kw, Q0 = cylinder_ns(N, nodes, viscous, ip)
    g, out, ref = residual_pair(orc, kw, perturbed(Q0, 0.02, seed=10 + N))
    assert rel_l2(out, ref) <= TOL_STAGE
    assert np.allclose(g.residuals(), np.abs(ref.reshape(-1, 4)).max(0), rtol=1e-11)


@pytest.mark.parametrize("wall,riemann", [("adiabatic", O.HLL), ("isothermal", O.LXF), ("isothermal", O.EXACT)])
def test_cylinder_ns_wall_types_and_fluxes(wall, riemann):
    orc, kw, Q0 = cylinder_ns(4, O.LG, O.BR1, wall=wall, riemann=riemann)
    _, out, ref = residual_pair(orc, kw, perturbed(Q0, 0.02, seed=3))
    assert rel_l2(out, ref) <= TOL_STAGE


@pytest.mark.parametrize("viscous,ip", [(O.BR1, 0), (O.IP, 0), (O.IP, 2)])
def test_periodic_ns_residual(viscous, ip):
    orc, kw, Q0 = vortex_ns(5, O.LGL, viscous, ip)
    _, out, ref = residual_pair(orc, kw, perturbed(Q0, 0.01, seed=4))
    assert rel_l2(out, ref) <= TOL_STAGE


@pytest.mark.parametrize("viscous", [O.BR1, O.IP])
def test_cylinder_ns_rk3_100_steps(viscous):
    orc, kw, Q0 = cylinder_ns(3, O.LGL, viscous)
    Q = perturbed(Q0, 0.01, seed=7)
    orc.set_state(Q)
    g = hg.GpuDGSEM(orc.export_mesh(), **kw)
    g.set_state(Q)
    dt = orc.estimate_dt(0.2, 1.0)
    assert abs(g.estimate_time_step(0.2, 1.0) - dt) <= 1e-14 * dt
    orc.time_step(O.RK3, 0.0, dt)
    g.time_step(hg.SCHEME_RK3, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STAGE
    for s in range(1, 100):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 99, dt, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_100
    np.testing.assert_allclose(g.residuals(), orc.residuals(), rtol=1e-9)


def test_ns_fp32_bulk_path():
    orc, kw, Q0 = cylinder_ns(4, O.LGL, O.BR1)
    Q = perturbed(Q0, 0.01, seed=8)
    g, out, ref = residual_pair(orc, kw, Q, precision=hg.PREC_FP32)
    assert rel_l2(out, ref) <= 1e-4
    g.set_state(Q)
    orc.set_state(Q)
    dt = orc.estimate_dt(0.2, 1.0)
    for s in range(20):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 20, 0.0, dt)
    rho_g, rho_o = g.state().reshape(-1, 4)[:, 0], orc.state().reshape(-1, 4)[:, 0]
    assert rel_l2(rho_g, rho_o) <= 1e-5


def test_ns_on_package_built_ogrid():
    """O-grid from the package's mesh builder (curved interior arcs) against the oracle's own construction."""
    m = hmesh.ogrid(6, 16, 0.5, 10.0, 1.2)
    obcs = [dict(type=O.BC_VISCOUSWALL, wall_type=2), dict(type=O.BC_FARFIELD)]
    orc = O.Oracle(m, 5, nodes=O.LG, riemann=O.ROE, mach=0.2, reynolds=100.0, navier_stokes=1, viscous=O.BR1,
                   bcs=obcs)
    q = dirichlet_state(orc, 0.2)
    kw = dict(mach=0.2, reynolds=100.0, navier_stokes=1, viscous=hg.BR1, node_type=hg.NODES_LG, riemann=hg.ROE,
              bcs=[dict(type=hg.BC_VISCOUSWALL, wall_type=2), dict(type=hg.BC_FARFIELD, state=q)])
    Q = perturbed(np.tile(q, orc.ndof // 4), 0.01, seed=9)
    _, out, ref = residual_pair(orc, kw, Q, mesh=hmesh.build_descriptor(m, 5, hg.NODES_LG))
    assert rel_l2(out, ref) <= TOL_STAGE


def test_zone_riemann_override_exact():
    """Roe inside, the exact solver on the Dirichlet and far-field zones (per-zone override)."""
    m = load_mesh("CylinderBench")
    T_ref = 273.15
    obcs = [dict(type=O.BC_DIRICHLET, riemann=O.EXACT), dict(type=O.BC_FARFIELD, riemann=O.EXACT),
            dict(type=O.BC_FARFIELD), dict(type=O.BC_PRESSUREOUTLET, outflow_type=2),
            dict(type=O.BC_VISCOUSWALL, wall_type=1, wall_T=1.1 * T_ref)]
    orc = O.Oracle(m, 3, nodes=O.LGL, riemann=O.ROE, mach=MACH, reynolds=RE, navier_stokes=1, viscous=O.BR1,
                   bcs=obcs)
    q = dirichlet_state(orc, MACH)
    gbcs = [dict(type=hg.BC_DIRICHLET, state=q, riemann=hg.EXACT), dict(type=hg.BC_FARFIELD, state=q, riemann=hg.EXACT),
            dict(type=hg.BC_FARFIELD, state=q), dict(type=hg.BC_PRESSUREOUTLET, state=q, outflow_type=2),
            dict(type=hg.BC_VISCOUSWALL, wall_type=1, wall_T=1.1)]
    kw = dict(mach=MACH, reynolds=RE, navier_stokes=1, viscous=hg.BR1, node_type=hg.NODES_LGL, riemann=hg.ROE,
              bcs=gbcs)
    _, out, ref = residual_pair(orc, kw, perturbed(np.tile(q, orc.ndof // 4), 0.02, seed=13))
    assert rel_l2(out, ref) <= TOL_STAGE


def test_zone_fed_per_node():
    """A Dirichlet zone fed per node (the reference's boundary-condition function; here a free stream
    with a varying density) against the oracle's per-node zone state, on the cylinder mesh with every
    other zone kind present; the states persist over RK steps, a second call replaces them."""
    orc, kw, Q0 = cylinder_ns(4, O.LG, O.BR1)
    Q = perturbed(Q0, 0.01, seed=12)
    Xb = orc.zone_edge_nodes(1)
    q = orc.zone_state(1)
    g = hg.GpuDGSEM(orc.export_mesh(), **kw)
    g.set_state(Q)
    before = g.compute_time_derivative(0.0)
    for amp in (0.05, -0.03):
        uB = (q[None, :] * (1.0 + amp * np.sin(3.0 * Xb[:, 0:1]) + 0.02 * Xb[:, 1:2] ** 2)).ravel()
        orc.set_zone_state(1, uB)
        orc.set_state(Q)
        ref = orc.time_derivative(0.0)
        g.set_boundary_state(1, uB)
        g.set_state(Q)
        out = g.compute_time_derivative(0.0)
        assert rel_l2(out, ref) <= TOL_STAGE
        assert rel_l2(before, ref) > 1e-8        # the per-node states change the residual
    dt = orc.estimate_dt(0.2, 1.0)
    for s in range(10):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 10, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STAGE * 10
    with pytest.raises(hg.HorsesGpuError):
        g.set_boundary_state(1, uB[:-4])          # wrong size
    with pytest.raises(hg.HorsesGpuError):
        g.set_boundary_state(2, np.zeros(orc.zone_edge_nodes(2).size * 2))   # far field: not fed per node
