"""Artificial dissipation across edges between orders and subdivided edges (DGSpatialDiscretizationMethods.f90:
603, 625 on interior edges, :816, 876-877 and :993, 1053-1054 on subdivided ones; DGArtificialDissipation.f90:
100-363): the jumps indicator sums each element's edge jumps at the edge's (half edges') own nodes, the edge
viscosity is the mean over the edge's two or three elements, and the Laplacian face term
-mu_a Area (qL - qR) (or, for the Physical type, mu + mu_a in the viscous fluxes and the penalty) enters the
mortar fluxes.  CUDA against the FP64 oracle on the same mesh and state: relative L2 <= 1e-12 per residual,
<= 1e-10 after RK steps, the element viscosities to 1e-12."""
import numpy as np
import pytest

from oracle import oracle as O
import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases as hcases
from cases_util import load_mesh, perturbed, rel_l2

pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-12
TOL_STEPS = 1e-10


def checker_av(viscous, av_type, ip_method=0, orders=(3, 5), n=5, re=200.0, intensity=0.5):
    """Periodic box of alternating orders (every interior edge between orders), Navier-Stokes with the
    jumps-based dissipation; the state carries a density step so that the indicator fires."""
    m = hmesh.cartesian(n, n, -5.0, 5.0, -5.0, 5.0)
    ij = np.arange(n * n)
    N = np.where((ij % n + ij // n) % 2 == 0, orders[0], orders[1])
    orc = O.Oracle(m, N, nodes=O.LG, riemann=O.ROE, mach=0.5, reynolds=re, navier_stokes=1, viscous=viscous,
                   ip_method=ip_method, sigma0_ip=5.0, bcs=hmesh.periodic_bcs_cartesian(), av_type=av_type,
                   av_intensity=intensity, av_indicator=O.IND_JUMPS)
    X = orc.coords()
    Q = hcases.isentropic_vortex(X[:, 0], X[:, 1], mach=0.5).reshape(-1, 4)
    Q[X[:, 0] > 1.3] *= 1.35        # density and energy step across a column of elements
    Q = perturbed(Q.ravel(), 0.01, seed=int(orders[1]) + viscous)
    g = hg.GpuDGSEM(orc.export_mesh(), mach=0.5, reynolds=re, navier_stokes=1, viscous=viscous, ip_method=ip_method,
                    sigma0_ip=5.0, node_type=hg.NODES_LG, riemann=hg.ROE, av_type=av_type, av_intensity=intensity,
                    bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    return orc, g, Q


@pytest.mark.parametrize("viscous,av_type,ip_method", [(O.IP, O.AV_LAPLACIAN, 0), (O.BR1, O.AV_LAPLACIAN, 0),
                                                       (O.IP, O.AV_PHYSICAL, 0), (O.IP, O.AV_LAPLACIAN, 2)])
def test_p_nonconforming_av(viscous, av_type, ip_method):
    # the Physical type puts mu_a into the viscous fluxes: a smaller intensity and step keep it explicit-stable
    phys = av_type == O.AV_PHYSICAL
    orc, g, Q = checker_av(viscous, av_type, ip_method, intensity=0.05 if phys else 0.5)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= TOL_STAGE
    mu_o = orc.av_viscosity()
    assert np.count_nonzero(mu_o) > 0                      # the step is flagged
    np.testing.assert_allclose(g.element_viscosity(), mu_o, rtol=1e-12, atol=1e-300)
    dt = (0.1 if phys else 0.5) * orc.estimate_dt(0.2, 1.0)
    for k in range(5):
        orc.time_step(O.RK3, k * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 5, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STEPS


def test_subdivided_edges_av():
    """CylinderRe1000 mesh (orders 4-10 by zone, edges between orders and 92 subdivided edges), SIPG,
    the jumps-based Laplacian dissipation, on a state with a density step across the wake."""
    m = load_mesh("CylinderInflation")
    porder = np.array([4, 6, 10, 8, 8])[m["p_zones"]]
    ex = O.EXACT
    bcs = [dict(type=O.BC_DIRICHLET, riemann=ex), dict(type=O.BC_DIRICHLET, riemann=ex),
           dict(type=O.BC_DIRICHLET, riemann=ex), dict(type=O.BC_PRESSUREOUTLET, outflow_type=2, riemann=ex),
           dict(type=O.BC_VISCOUSWALL, wall_type=2, riemann=ex)]
    orc = O.Oracle(m, porder, nodes=O.LG, riemann=O.HLL, mach=0.1, reynolds=1000.0, prandtl=0.72, navier_stokes=1,
                   viscous=O.IP, ip_method=0, sigma0_ip=10.0, bcs=bcs, av_type=O.AV_LAPLACIAN, av_intensity=0.4,
                   av_indicator=O.IND_JUMPS)
    r = orc.ref
    cv = 287.15 * 2.5
    q = np.array([r["rho"], r["rho"] * r["V"], 0.0, cv * r["rho"] * r["T"] + 0.5 * r["rho"] * r["V"] * r["V"]])
    q = q / np.array([r["rho"], r["rho"] * r["a"], r["rho"] * r["a"], r["p"]])
    X = orc.coords()
    Q = np.tile(q, (len(X), 1))
    Q[X[:, 0] > 0.8] *= 1.2
    Q = perturbed(Q.ravel(), 0.01, seed=51)
    ge = hg.EXACT
    zq = [orc.zone_state(z) for z in range(1, 5)]
    gbcs = [dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[0]), dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[1]),
            dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[2]),
            dict(type=hg.BC_PRESSUREOUTLET, outflow_type=2, riemann=ge, state=zq[3]),
            dict(type=hg.BC_VISCOUSWALL, wall_type=2, riemann=ge)]
    g = hg.GpuDGSEM(orc.export_mesh(), mach=0.1, reynolds=1000.0, prandtl=0.72, navier_stokes=1, viscous=hg.IP,
                    ip_method=hg.SIPG, sigma0_ip=10.0, node_type=hg.NODES_LG, riemann=hg.HLL, bcs=gbcs,
                    av_type=hg.AV_LAPLACIAN, av_intensity=0.4)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= TOL_STAGE
    mu_o = orc.av_viscosity()
    assert np.count_nonzero(mu_o) > 0
    np.testing.assert_allclose(g.element_viscosity(), mu_o, rtol=1e-12, atol=1e-300)
    dt = orc.estimate_dt(0.1, 1e-2)
    for k in range(3):
        orc.time_step(O.RK5, k * dt, dt)
    g.time_steps(hg.SCHEME_RK5, 3, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STEPS
