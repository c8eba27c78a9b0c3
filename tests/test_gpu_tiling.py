"""Elements-per-CTA variants of the stage kernels and the autotuner that picks one.

Every variant must give the oracle's residual (FP64: relative L2 <= 1e-12) and RK3 steps
(<= 1e-11 after 10 steps) on Euler (LG and LGL, Roe and the exact solver), Navier-Stokes (BR1, IP)
and artificial dissipation with the learned sensor (network inference inside the gradient kernel
with one element per CTA).  hg_autotune must pick a variant, leave the state unchanged and leave the
residual of the resident state for hg_residuals.
"""
import numpy as np
import pytest

from oracle import oracle as O
import horses2d_b200 as hg
from cases_util import vortex_case, perturbed, rel_l2

pytestmark = pytest.mark.gpu


def check_variants(orc, make, Q, steps=10, cfl=0.2, tol=1e-12):
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    dt = orc.estimate_dt(cfl, 1.0)
    for s in range(steps):
        orc.time_step(O.RK3, s * dt, dt)
    ref_steps = orc.state()
    for v in range(hg.lib.TILINGS):
        g = make()
        g.set_tiling(v)
        assert g.get_tiling()["variant"] == v
        g.set_state(Q)
        assert rel_l2(g.compute_time_derivative(0.0), ref) <= tol, v
        g.time_steps(hg.SCHEME_RK3, steps, 0.0, dt)
        assert rel_l2(g.state(), ref_steps) <= 10 * tol, v
        g.close()


@pytest.mark.parametrize("nodes,N,riemann", [(O.LGL, 4, O.ROE), (O.LG, 3, O.EXACT), (O.LGL, 7, O.HLL)])
def test_euler_variants(nodes, N, riemann):
    orc, Q0, prm = vortex_case(n=8, N=N, nodes=nodes, riemann=riemann)
    mesh = orc.export_mesh()
    check_variants(orc, lambda: hg.GpuDGSEM(mesh, mach=prm["mach"], node_type=prm["node_type"],
                                            riemann=prm["riemann"], bcs=prm["bcs"]), perturbed(Q0, 0.02, seed=N))


@pytest.mark.parametrize("viscous,ip", [(O.BR1, 0), (O.IP, 0)])
def test_navier_stokes_variants(viscous, ip):
    from test_gpu_ns_parity import cylinder_ns
    orc, kw, Q0 = cylinder_ns(5, O.LG, viscous, ip)
    mesh = orc.export_mesh()
    check_variants(orc, lambda: hg.GpuDGSEM(mesh, **kw), perturbed(Q0, 0.01, seed=31), cfl=0.05)


def test_learned_sensor_variants():
    from test_gpu_sensor import small_shock, random_problem
    orc, g0, Q = small_shock(indicator=O.IND_EXTERNAL, sensor=hg.SENSOR_LEARNED)
    p, _, _, _ = random_problem(1, 7)
    g0.set_sensor(hg.SENSOR_LEARNED, mlp=p)
    g0.set_state(Q)
    _, out = g0.sensor_eval()
    orc.set_av_g(out[:, 3])
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    for v in range(hg.lib.TILINGS):
        g0.set_tiling(v)
        g0.set_state(Q)
        assert rel_l2(g0.compute_time_derivative(0.0), ref) <= 1e-12, v


def test_autotune_keeps_state_and_residual():
    orc, Q0, prm = vortex_case(n=8, N=4, nodes=O.LGL, riemann=O.ROE)
    Q = perturbed(Q0, 0.02, seed=3)
    g = hg.GpuDGSEM(orc.export_mesh(), mach=prm["mach"], node_type=prm["node_type"], riemann=prm["riemann"],
                    bcs=prm["bcs"])
    g.set_state(Q)
    r = g.autotune(trials=5)
    assert r["chosen"] in range(hg.lib.TILINGS) and r["tiling"]["variant"] == r["chosen"]
    assert all(ms > 0.0 for ms in r["ms"])
    assert np.array_equal(g.state(), Q)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    np.testing.assert_allclose(g.residuals(), np.abs(ref.reshape(-1, 4)).max(0), rtol=1e-11)
    t = g.get_tiling()
    assert t["elements_per_cta"] >= 1 and t["threads_per_cta"] % 32 == 0
    with pytest.raises(hg.HorsesGpuError):
        g.set_tiling(hg.lib.TILINGS)


def test_autotune_of_a_fused_ip_context_leaves_it_as_set_state_does():
    """The autotuner times RK3 steps with dt = 0 and puts the state back; a fused interior-penalty context
    with the modal indicator (gradient traces and indicator formed in the stage epilogues) then steps
    exactly as a context that was only given the state, in the same tiling."""
    from horses2d_b200 import mesh as hmesh, cases
    n, N = 12, 5
    m = hmesh.cartesian(n, n, 0.0, 1.0, 0.0, 1.0)
    orc = O.Oracle(m, N, nodes=O.LG, riemann=O.ROE, mach=0.3, reynolds=1.0e4, navier_stokes=1, viscous=O.IP,
                   ip_method=0, sigma0_ip=10.0, bcs=hmesh.periodic_bcs_cartesian())
    X = orc.coords()
    Q = perturbed(cases.kelvin_helmholtz(X[:, 0], X[:, 1], seed=5).ravel(), 1e-3, seed=6)

    def ctx():
        g = hg.GpuDGSEM(orc.export_mesh(), mach=0.3, reynolds=1.0e4, navier_stokes=1, viscous=hg.IP,
                        ip_method=hg.SIPG, sigma0_ip=10.0, node_type=hg.NODES_LG, riemann=hg.ROE,
                        av_type=hg.AV_LAPLACIAN, av_intensity=1.0, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
        g.set_sensor(hg.SENSOR_MODAL)
        g.set_state(Q)
        return g

    a, b = ctx(), ctx()
    r = a.autotune(trials=3)
    assert np.array_equal(a.state(), Q)
    b.set_tiling(r["chosen"])
    dt = 0.05 / n ** 2
    for s in range(3):
        a.time_step(hg.SCHEME_RK3, s * dt, dt)
        b.time_step(hg.SCHEME_RK3, s * dt, dt)
    assert np.array_equal(a.state(), b.state())
    np.testing.assert_array_equal(a.element_viscosity(), b.element_viscosity())
