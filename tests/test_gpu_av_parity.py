"""GPU parity of the artificial dissipation (jumps-based indicator, Laplacian and Physical types) and of
the newDirichlet zone, against the FP64 oracle (which reproduces the reference's Ramp benchmark).

State: the Ramp case (Mach 2, Re = 0, N = 3, Legendre-Gauss) after 300 oracle RK5 iterations from the
uniform state, so the compression corner has formed and the indicator is active.
FP64 tolerances: relative L2 <= 1e-12 per residual, <= 1e-10 after 50 RK3 steps.
"""
import numpy as np
import pytest

from oracle import oracle as O
import horses2d_b200 as hg
from cases_util import rel_l2, load_mesh, dirichlet_state

pytestmark = pytest.mark.gpu


def ramp(viscous=O.IP, ip_method=2, av_type=O.AV_LAPLACIAN, intensity=0.1, iters=300):
    bcs = [dict(type=O.BC_EULERWALL), dict(type=O.BC_EULERWALL), dict(type=O.BC_NEWDIRICHLET),
           dict(type=O.BC_NEWDIRICHLET)]
    kw = dict(nodes=O.LG, riemann=O.ROE, mach=2.0, reynolds=0.0, prandtl=0.72, navier_stokes=1, viscous=viscous,
              ip_method=ip_method, sigma0_ip=1.0, bcs=bcs, av_type=av_type, av_intensity=intensity)
    orc = O.Oracle(load_mesh("RampBench"), 3, **kw)
    r = orc.ref
    cv = 287.15 * 2.5
    q = np.array([r["rho"], r["rho"] * r["V"], 0.0, cv * r["rho"] * r["T"] + 0.5 * r["rho"] * r["V"] * r["V"]])
    q = q / np.array([r["rho"], r["rho"] * r["a"], r["rho"] * r["a"], r["p"]])
    orc.set_state(np.tile(q, orc.ndof // 4))
    if iters:
        orc.integrate(O.RK5, transient=False, t0=0.0, t_end=1.0, max_iter=iters, cfl=0.1, dt_cap=2.0,
                      residual_target=1e-12)
    qz = dirichlet_state(orc, 2.0)
    gkw = dict(mach=2.0, reynolds=0.0, prandtl=0.72, navier_stokes=1, viscous=viscous, ip_method=ip_method,
               sigma0_ip=1.0, node_type=hg.NODES_LG, riemann=hg.ROE, av_type=av_type, av_intensity=intensity,
               bcs=[dict(type=hg.BC_EULERWALL), dict(type=hg.BC_EULERWALL),
                    dict(type=hg.BC_NEWDIRICHLET, state=qz), dict(type=hg.BC_NEWDIRICHLET, state=qz)])
    return orc, gkw, orc.state()


@pytest.mark.parametrize("viscous,ip,av", [(O.IP, 2, O.AV_LAPLACIAN), (O.IP, 0, O.AV_LAPLACIAN),
                                           (O.BR1, 0, O.AV_LAPLACIAN), (O.IP, 2, O.AV_PHYSICAL),
                                           (O.BR1, 0, O.AV_PHYSICAL)])
def test_ramp_residual_with_artificial_dissipation(viscous, ip, av):
    orc, gkw, Q = ramp(viscous, ip, av)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = hg.GpuDGSEM(orc.export_mesh(), **gkw)
    g.set_state(Q)
    out = g.compute_time_derivative(0.0)
    assert rel_l2(out, ref) <= 1e-12
    # the dissipation is active on this state: switching it off changes the residual
    orc_off, _, _ = ramp(viscous, ip, O.AV_NONE, iters=0)
    orc_off.set_state(Q)
    assert rel_l2(orc_off.time_derivative(0.0), ref) > 1e-6


def test_ramp_rk3_steps_with_laplacian_dissipation():
    _, gkw, Q = ramp()
    orc, _, _ = ramp(iters=0)   # a fresh oracle: the dt estimate keeps running maxima (SAVE) across calls
    orc.set_state(Q)
    g = hg.GpuDGSEM(orc.export_mesh(), **gkw)
    g.set_state(Q)
    dt = orc.estimate_dt(0.1, 2.0)
    assert abs(g.estimate_time_step(0.1, 2.0) - dt) <= 1e-14 * dt
    for s in range(50):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 50, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= 1e-10
    np.testing.assert_allclose(g.residuals(), orc.residuals(), rtol=1e-9)


def test_newdirichlet_total_pressure_mode():
    """newDirichlet 'Specify total pressure' inflow and total outflow pressure, Euler-like NS build."""
    orc, gkw, Q = ramp(iters=100)
    bcs = [dict(type=O.BC_EULERWALL), dict(type=O.BC_EULERWALL),
           dict(type=O.BC_NEWDIRICHLET, mode=1, outflow_total=1, mach=0.5),
           dict(type=O.BC_NEWDIRICHLET, mode=1, outflow_total=1, mach=0.5)]
    orc2 = O.Oracle(load_mesh("RampBench"), 3, nodes=O.LG, riemann=O.ROE, mach=2.0, reynolds=0.0, navier_stokes=1,
                    viscous=O.IP, ip_method=2, bcs=bcs, av_type=O.AV_LAPLACIAN, av_intensity=0.1)
    qz = dirichlet_state(orc2, 0.5)
    gkw["bcs"] = [dict(type=hg.BC_EULERWALL), dict(type=hg.BC_EULERWALL),
                  dict(type=hg.BC_NEWDIRICHLET, state=qz, mode=1, outflow_total=1),
                  dict(type=hg.BC_NEWDIRICHLET, state=qz, mode=1, outflow_total=1)]
    # a subsonic state: the free stream at Mach 0.5 with a perturbation
    rng = np.random.default_rng(5)
    Qs = np.tile(qz, orc2.ndof // 4) * (1.0 + 0.01 * rng.standard_normal(orc2.ndof))
    orc2.set_state(Qs)
    ref = orc2.time_derivative(0.0)
    g = hg.GpuDGSEM(orc2.export_mesh(), **gkw)
    g.set_state(Qs)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= 1e-12


@pytest.mark.parametrize("precision", [hg.PREC_FP64, hg.PREC_FP32])
def test_shear_layer_n7_sipg_modal_dissipation(precision):
    """The Kelvin-Helmholtz workload's physics at a small size: periodic 8 x 8, N = 7, Re 1e4, M 0.3,
    SIPG (sigma0 10), Roe, Laplacian artificial viscosity driven by the modal indicator (a density
    contrast across thin layers, so that some elements are flagged); residual and 10 RK3 steps against
    the oracle, with the workload's step rule dt = min(CFL 0.2 estimate, 0.05 / n^2)."""
    from horses2d_b200 import mesh as hmesh, cases
    m = hmesh.cartesian(8, 8, 0.0, 1.0, 0.0, 1.0)
    orc = O.Oracle(m, 7, nodes=O.LG, riemann=O.ROE, mach=0.3, reynolds=1.0e4, navier_stokes=1, viscous=O.IP,
                   ip_method=0, sigma0_ip=10.0, bcs=hmesh.periodic_bcs_cartesian(), av_type=O.AV_LAPLACIAN,
                   av_intensity=1.0, av_indicator=O.IND_MODAL)
    X = orc.coords()
    Q = cases.kelvin_helmholtz(X[:, 0], X[:, 1], delta=0.005, eps=0.05, seed=5, drho=2.0).ravel()
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    assert np.max(orc.av_viscosity()) > 0.0
    g = hg.GpuDGSEM(orc.export_mesh(), precision=precision, mach=0.3, reynolds=1.0e4, navier_stokes=1,
                    viscous=hg.IP, ip_method=hg.SIPG, sigma0_ip=10.0, node_type=hg.NODES_LG, riemann=hg.ROE,
                    av_type=hg.AV_LAPLACIAN, av_intensity=1.0, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    g.set_sensor(hg.SENSOR_MODAL)
    g.set_state(Q)
    fp64 = precision == hg.PREC_FP64
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= (1e-12 if fp64 else 1e-4)
    np.testing.assert_allclose(g.element_viscosity(), orc.av_viscosity(), rtol=1e-12 if fp64 else 1e-4, atol=1e-300)
    dt = min(orc.estimate_dt(0.2, 1.0), 0.05 / 8 ** 2)
    for s in range(10):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 10, 0.0, dt)
    if fp64:
        assert rel_l2(g.state(), orc.state()) <= 1e-10
    else:
        # this 8 x 8 case is under-resolved on purpose (the layers must trip the indicator) and its
        # residual grows ~20x over the 10 steps, which amplifies FP32 rounding: 5e-5 here; the
        # workload-size FP32 density error is reported by bench.py
        assert rel_l2(g.state()[0::4], orc.state()[0::4]) <= 5e-5
