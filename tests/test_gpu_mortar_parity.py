"""GPU parity on meshes with mixed polynomial orders and subdivided edges (Euler build).

Projection types 3-6 (an edge between two orders, evaluated at the higher one) and the mortars of
subdivided edges run in the mortar kernel; every order keeps its own fused stage kernel.  Checked
against the FP64 oracle: relative L2 <= 1e-12 per residual, <= 1e-10 after RK steps; the FP32 bulk
path <= 1e-5 (density).  The VortexTransport benchmark (curved, N = 5/7/12, 34 subdivided edges,
periodic) runs end to end: the reference's iteration count and max-norm errors.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases as hcases
from cases_util import GOLDEN, load_mesh, perturbed, rel_l2
from test_oracle import vortex_transport_ic, vortex_transport_oracle

pytestmark = pytest.mark.gpu

TOL_STAGE = 1e-12
TOL_STEPS = 1e-10


def gpu_from(orc, mach, nodes, riemann, bcs, precision=hg.PREC_FP64):
    return hg.GpuDGSEM(orc.export_mesh(), mach=mach, node_type=nodes, riemann=riemann, bcs=bcs, precision=precision)


def periodic_gpu_bcs():
    return [dict(type=hg.BC_PERIODIC)] * 4


def vt_bcs():
    return [dict(type=hg.BC_PERIODIC)] * 4


def checker_case(nodes, riemann, orders=(3, 5), n=5):
    """Periodic box whose elements alternate between two orders: every interior edge is p-nonconforming
    (odd n: periodic partners share an order)."""
    m = hmesh.cartesian(n, n, -5.0, 5.0, -5.0, 5.0)
    ij = np.arange(n * n)
    N = np.where((ij % n + ij // n) % 2 == 0, orders[0], orders[1])
    orc = O.Oracle(m, N, nodes=nodes, riemann=riemann, mach=0.5, bcs=hmesh.periodic_bcs_cartesian())
    X = orc.coords()
    Q = perturbed(hcases.isentropic_vortex(X[:, 0], X[:, 1], mach=0.5).ravel(), 0.02, seed=int(orders[1]))
    return orc, Q


@pytest.mark.parametrize("nodes,riemann,orders", [(O.LG, O.ROE, (3, 5)), (O.LGL, O.HLL, (2, 4)),
                                                  (O.LG, O.EXACT, (4, 6)), (O.LGL, O.LXF, (5, 8))])
def test_p_nonconforming_residual(nodes, riemann, orders):
    orc, Q = checker_case(nodes, riemann, orders)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = gpu_from(orc, 0.5, nodes, riemann, periodic_gpu_bcs())
    g.set_state(Q)
    assert np.array_equal(g.state(), Q)
    out = g.compute_time_derivative(0.0)
    assert rel_l2(out, ref) <= TOL_STAGE
    np.testing.assert_allclose(g.residuals(), np.abs(ref.reshape(-1, 4)).max(0), rtol=1e-11)


@pytest.mark.parametrize("scheme", [hg.SCHEME_RK3, hg.SCHEME_RK5])
def test_p_nonconforming_steps(scheme):
    orc, Q = checker_case(O.LG, O.ROE, (3, 5))
    g = gpu_from(orc, 0.5, O.LG, O.ROE, periodic_gpu_bcs())
    orc.set_state(Q)
    g.set_state(Q)
    dt = 2e-3
    for k in range(3):
        orc.time_step(scheme, k * dt, dt)
    g.time_steps(scheme, 3, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STEPS
    # the graph path (pairs of steps)
    for k in range(3, 13):
        orc.time_step(scheme, k * dt, dt)
    g.time_steps(scheme, 10, 3 * dt, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STEPS


@pytest.mark.parametrize("uniform", [False, True])
def test_vortex_transport_mesh_residual(uniform):
    """Curved mesh with 34 subdivided edges (hanging nodes) and periodic zones; N = 5/7/12 by zone, or
    one order everywhere (mortars alone)."""
    if uniform:
        m = load_mesh("VortexTransportBench")
        bcs = [dict(type=O.BC_PERIODIC, periodic_dir=2, connected_marker=2),
               dict(type=O.BC_PERIODIC, periodic_dir=2, connected_marker=1),
               dict(type=O.BC_PERIODIC, periodic_dir=1, connected_marker=4),
               dict(type=O.BC_PERIODIC, periodic_dir=1, connected_marker=3)]
        orc = O.Oracle(m, 4, nodes=O.LG, riemann=O.ROE, mach=0.6, reynolds=0.0, bcs=bcs)
    else:
        orc = vortex_transport_oracle()
    X = orc.coords()
    Q = perturbed(vortex_transport_ic(X, orc.ref).ravel(), 0.01, seed=5)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = gpu_from(orc, 0.6, O.LG, O.ROE, vt_bcs())
    g.set_state(Q)
    out = g.compute_time_derivative(0.0)
    assert rel_l2(out, ref) <= TOL_STAGE
    dt = 1e-3
    for k in range(5):
        orc.time_step(O.RK5, k * dt, dt)
    g.time_steps(hg.SCHEME_RK5, 5, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STEPS


def test_vortex_transport_fp32():
    """FP32 bulk arithmetic on the mortar mesh: the residual of a perturbed state to the FP32 bound
    (relative 1e-4), and the stepped density of the vortex within the 1e-5 relative L2 target."""
    orc = vortex_transport_oracle()
    X = orc.coords()
    Q0 = vortex_transport_ic(X, orc.ref).ravel()
    Q = perturbed(Q0, 0.02, seed=9)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = gpu_from(orc, 0.6, O.LG, O.ROE, vt_bcs(), precision=hg.PREC_FP32)
    g.set_state(Q)
    out = g.compute_time_derivative(0.0)
    assert rel_l2(out, ref) <= 1e-4
    orc.set_state(Q0)
    g.set_state(Q0)
    dt = orc.estimate_dt(0.4, 1e-2)
    for s in range(20):
        orc.time_step(O.RK5, s * dt, dt)
    g.time_steps(hg.SCHEME_RK5, 20, 0.0, dt)
    assert rel_l2(g.state().reshape(-1, 4)[:, 0], orc.state().reshape(-1, 4)[:, 0]) <= 1e-5


def test_vortex_transport_benchmark_golden():
    """The reference's VortexTransport regression (TestCases/Benchmark/Simulations/VortexTransport):
    Williamson RK5, CFL 0.4, dt cap 1e-2, transient to t = 2; the reference asserts the iteration
    count and the four max-norm errors against the initial vortex (to 1e-12).  On the device the run
    takes the same dt sequence (same iteration count); the errors agree to 1e-10."""
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["VortexTransport"]
    orc = vortex_transport_oracle()
    X = orc.coords()
    Q0 = vortex_transport_ic(X, orc.ref).ravel()
    g = gpu_from(orc, 0.6, O.LG, O.ROE, vt_bcs())
    g.set_state(Q0)
    it, t = g.integrate(hg.SCHEME_RK5, transient=True, t0=0.0, t_end=2.0, max_iter=1000000, cfl=0.4, dt_cap=1e-2)
    assert it == golden["expected_iter"]
    assert t == pytest.approx(2.0, abs=1e-14)
    err = np.abs(Q0.reshape(-1, 4) - g.state().reshape(-1, 4)).max(0)
    assert np.max(np.abs(err - np.array(golden["expectedErrors"]))) <= 1e-10


def test_composite_monitors_and_restart(tmp_path):
    """State round trip, probes and restart files through the composite context."""
    orc, Q = checker_case(O.LG, O.ROE, (3, 5))
    g = gpu_from(orc, 0.5, O.LG, O.ROE, periodic_gpu_bcs())
    g.set_state(Q)
    g.time_steps(hg.SCHEME_RK3, 4, 0.0, 1e-3)
    orc.set_state(Q)
    for k in range(4):
        orc.time_step(O.RK3, k * 1e-3, 1e-3)
    els = np.array([0, 1, 7, 19], np.int32)
    xe = np.array([[0.3, 0.6], [0.1, 0.9], [0.5, 0.5], [0.77, 0.2]])
    got = g.probes(els, xe)
    for k in range(len(els)):
        np.testing.assert_allclose(got[k], orc.probe(int(els[k]), *xe[k]), rtol=1e-10, atol=1e-12)
    p = tmp_path / "mixed.HiORst"
    g.save_restart(p, 4e-3, 4)
    h = gpu_from(orc, 0.5, O.LG, O.ROE, periodic_gpu_bcs())
    t, it = h.load_restart(p)
    assert (t, it) == (4e-3, 4) and np.array_equal(h.state(), g.state())
    assert g.autotune(3)["chosen"] in (0, 1)
    g.time_steps(hg.SCHEME_RK3, 2, 4e-3, 1e-3)
    h.time_steps(hg.SCHEME_RK3, 2, 4e-3, 1e-3)
    assert np.array_equal(g.state(), h.state())


# ----------------------------------------------------------------------------- Navier-Stokes (BR1)
def cylinder_re100_case(orders=(8, 2, 8, 6, 4)):
    m = load_mesh("CylinderBench")
    porder = np.array(orders)[m["p_zones"]]
    ex = O.EXACT
    bcs = [dict(type=O.BC_DIRICHLET, riemann=ex), dict(type=O.BC_DIRICHLET, riemann=ex),
           dict(type=O.BC_DIRICHLET, riemann=ex), dict(type=O.BC_PRESSUREOUTLET, outflow_type=2, riemann=ex),
           dict(type=O.BC_VISCOUSWALL, wall_type=2, riemann=ex)]
    orc = O.Oracle(m, porder, nodes=O.LG, riemann=O.HLL, mach=0.1, reynolds=100.0, prandtl=0.72, navier_stokes=1,
                   viscous=O.BR1, bcs=bcs)
    r = orc.ref
    cv = 287.15 * 2.5
    q = np.array([r["rho"], r["rho"] * r["V"], 0.0, cv * r["rho"] * r["T"] + 0.5 * r["rho"] * r["V"] * r["V"]])
    q = q / np.array([r["rho"], r["rho"] * r["a"], r["rho"] * r["a"], r["p"]])
    ge = hg.EXACT
    zq = [orc.zone_state(z) for z in range(1, 5)]
    gbcs = [dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[0]), dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[1]),
            dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[2]),
            dict(type=hg.BC_PRESSUREOUTLET, outflow_type=2, riemann=ge, state=zq[3]),
            dict(type=hg.BC_VISCOUSWALL, wall_type=2, riemann=ge)]
    kw = dict(mach=0.1, reynolds=100.0, prandtl=0.72, navier_stokes=1, viscous=hg.BR1, node_type=hg.NODES_LG,
              riemann=hg.HLL, bcs=gbcs)
    return orc, q, kw


def test_ns_p_nonconforming_residual():
    """CylinderRe100 mesh, orders 2-8 by zone (112 edges between orders), BR1, HLL, exact solver on
    the zones: residual of a perturbed state and RK5 steps."""
    orc, q, kw = cylinder_re100_case()
    Q = perturbed(np.tile(q, orc.ndof // 4), 0.01, seed=31)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = hg.GpuDGSEM(orc.export_mesh(), **kw)
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= TOL_STAGE
    dt = orc.estimate_dt(0.1, 1e-2)    # the benchmark's CFL (order 8 elements near the wall)
    for k in range(4):
        orc.time_step(O.RK5, k * dt, dt)
    g.time_steps(hg.SCHEME_RK5, 4, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STEPS


def couette_case():
    """The Couette benchmark's set-up (TestCases/Benchmark/Simulations/Couette): curved mesh with 34
    subdivided edges, orders 5/7/10/7 by zone, BR1, Roe, isothermal walls (one moving), a Dirichlet
    zone fed by the plugin's boundary-condition function, a partially non-reflective outlet."""
    from test_oracle import couette_state
    m = load_mesh("CouetteBench")
    porder = np.array([5, 7, 10, 7])[m["p_zones"]]
    bcs = [dict(type=O.BC_VISCOUSWALL, wall_type=1),
           dict(type=O.BC_VISCOUSWALL, wall_type=1, wall_v=(np.sqrt(1.4) * 0.8, 0.0)),
           dict(type=O.BC_DIRICHLET), dict(type=O.BC_PRESSUREOUTLET, outflow_type=2)]
    orc = O.Oracle(m, porder, nodes=O.LG, riemann=O.ROE, mach=0.8, reynolds=2000.0, prandtl=0.72,
                   navier_stokes=1, viscous=O.BR1, bcs=bcs)
    ref = orc.ref
    scale = np.array([ref["rho"], ref["rho"] * ref["a"], ref["rho"] * ref["a"], ref["p"]])
    X = orc.coords()
    Q = perturbed((couette_state(X[:, 0], X[:, 1], ref) / scale).ravel(), 0.01, seed=32)
    Xb = orc.zone_edge_nodes(3)
    uB = (couette_state(Xb[:, 0], Xb[:, 1], ref) / scale).ravel()
    orc.set_zone_state(3, uB)
    q0 = couette_state(X[:, 0], X[:, 1], ref)
    q0[X[:, 0] ** 2 + X[:, 1] ** 2 < 0.005, 1] *= 1.005
    gbcs = [dict(type=hg.BC_VISCOUSWALL, wall_type=1, wall_T=1.0),
            dict(type=hg.BC_VISCOUSWALL, wall_type=1, wall_T=1.0, wall_v=(np.sqrt(1.4) * 0.8, 0.0)),
            dict(type=hg.BC_DIRICHLET, state=orc.zone_state(3)),
            dict(type=hg.BC_PRESSUREOUTLET, outflow_type=2, state=orc.zone_state(4))]
    g = hg.GpuDGSEM(orc.export_mesh(), mach=0.8, reynolds=2000.0, prandtl=0.72, navier_stokes=1, viscous=hg.BR1,
                    node_type=hg.NODES_LG, riemann=hg.ROE, bcs=gbcs)
    g.set_boundary_state(3, uB)
    return orc, g, Q, (q0 / scale).ravel()


def test_ns_subdivided_edges_residual():
    orc, g, Q, _ = couette_case()
    orc.set_state(Q)
    qd = orc.time_derivative(0.0)
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), qd) <= TOL_STAGE
    dt = orc.estimate_dt(0.4, 1.0)
    for k in range(4):
        orc.time_step(O.RK5, k * dt, dt)
    g.time_steps(hg.SCHEME_RK5, 4, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STEPS


def test_couette_benchmark_golden():
    """The reference's Couette regression on the device: steady RK5 at CFL 0.4 until the largest
    residual drops below 1e-4; the reference asserts iteration 19585 and the four final residuals
    (to 1e-12)."""
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["Couette"]
    _, g, _, Q0 = couette_case()
    g.set_state(Q0)
    it, _ = g.integrate(hg.SCHEME_RK5, transient=False, t0=0.0, t_end=1.0, max_iter=100000, cfl=0.4, dt_cap=1.0,
                        residual_target=1e-4)
    assert it == golden["expected_iter"]
    assert np.max(np.abs(g.residuals() - np.array(golden["expectedResiduals"]))) <= 1e-12


def test_cylinder_re100_benchmark_golden():
    """The reference's CylinderRe100 regression on the device: 250 steady RK5 iterations (CFL 0.1, dt
    cap 1e-2) on the p-refined cylinder mesh; final residuals and the wall's lift and drag."""
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["CylinderRe100"]
    orc, q, kw = cylinder_re100_case()
    g = hg.GpuDGSEM(orc.export_mesh(), **kw)
    g.set_state(np.tile(q, orc.ndof // 4))
    it, _ = g.integrate(hg.SCHEME_RK5, transient=False, t0=0.0, t_end=1e9, max_iter=250, cfl=0.1, dt_cap=1e-2,
                        residual_target=1e-14)
    assert it == 250
    np.testing.assert_allclose(g.residuals(), golden["residuals"], rtol=1e-9)
    r = orc.ref
    si = g.surface_integrals(5)
    dyn = 0.5 * r["rho"] * r["V"] * r["V"] * 1.0
    force = (si["pressure_force"] - si["viscous_force"] * np.sqrt(1.4) * 0.1) * r["p"] * r["L"]
    assert abs(force[1] / dyn - golden["cl"]) <= 1e-12
    assert abs(force[0] / dyn - golden["cd"]) <= 5e-8


def test_ns_p_nonconforming_fp32():
    """FP32 bulk path of the Navier-Stokes composite (CylinderRe100 mesh): residual to the FP32 bound,
    and the stepped density within the 1e-5 relative L2 target."""
    orc, q, kw = cylinder_re100_case()
    Q = perturbed(np.tile(q, orc.ndof // 4), 0.01, seed=33)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g = hg.GpuDGSEM(orc.export_mesh(), precision=hg.PREC_FP32, **kw)
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= 1e-4
    dt = orc.estimate_dt(0.1, 1e-2)
    for k in range(10):
        orc.time_step(O.RK5, k * dt, dt)
    g.time_steps(hg.SCHEME_RK5, 10, 0.0, dt)
    assert rel_l2(g.state().reshape(-1, 4)[:, 0], orc.state().reshape(-1, 4)[:, 0]) <= 1e-5


# ----------------------------------------------------------------------------- Navier-Stokes (interior penalty)
def cylinder_re1000_gpu(ip_method=0):
    from test_oracle import cylinder_re1000_oracle
    orc, q = cylinder_re1000_oracle(ip_method)
    ge = hg.EXACT
    zq = [orc.zone_state(z) for z in range(1, 5)]
    gbcs = [dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[0]), dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[1]),
            dict(type=hg.BC_DIRICHLET, riemann=ge, state=zq[2]),
            dict(type=hg.BC_PRESSUREOUTLET, outflow_type=2, riemann=ge, state=zq[3]),
            dict(type=hg.BC_VISCOUSWALL, wall_type=2, riemann=ge)]
    g = hg.GpuDGSEM(orc.export_mesh(), mach=0.1, reynolds=1000.0, prandtl=0.72, navier_stokes=1, viscous=hg.IP,
                    ip_method=ip_method, sigma0_ip=10.0, node_type=hg.NODES_LG, riemann=hg.HLL, bcs=gbcs)
    return orc, q, g


@pytest.mark.parametrize("ip_method", [hg.NIPG, hg.IIPG])
def test_ns_ip_variants_mortar_residual(ip_method):
    """NIPG (epsilon = +1) and IIPG (no gradient-face terms) through the mortars: residual parity."""
    orc, q, g = cylinder_re1000_gpu(ip_method)
    Q = perturbed(np.tile(q, orc.ndof // 4), 0.01, seed=42 + ip_method)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= TOL_STAGE


def test_ns_ip_mortar_residual():
    """CylinderRe1000 mesh (orders 4-10, 138 edges between orders, 92 subdivided edges), SIPG: the
    penalty at the edge's order and the gradient-face terms through the mortars; residual of a
    perturbed state and RK5 steps."""
    orc, q, g = cylinder_re1000_gpu()
    Q = perturbed(np.tile(q, orc.ndof // 4), 0.01, seed=41)
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g.set_state(Q)
    assert rel_l2(g.compute_time_derivative(0.0), ref) <= TOL_STAGE
    dt = orc.estimate_dt(0.1, 1e-2)
    for k in range(3):
        orc.time_step(O.RK5, k * dt, dt)
    g.time_steps(hg.SCHEME_RK5, 3, 0.0, dt)
    assert rel_l2(g.state(), orc.state()) <= TOL_STEPS


def test_cylinder_re1000_benchmark_golden():
    """The reference's CylinderRe1000 regression on the device: transient RK5 to t = 0.013 (CFL 0.1,
    dt cap 1e-2); iteration 512, the final residuals (reference: 1e-10) and the wall's lift and drag."""
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["CylinderRe1000"]
    orc, q, g = cylinder_re1000_gpu()
    g.set_state(np.tile(q, orc.ndof // 4))
    it, _ = g.integrate(hg.SCHEME_RK5, transient=True, t0=0.0, t_end=0.013, max_iter=10000000, cfl=0.1, dt_cap=1e-2)
    assert it == golden["expected_iter"]
    np.testing.assert_allclose(g.residuals(), golden["residuals"], rtol=1e-9)
    r = orc.ref
    si = g.surface_integrals(5)
    dyn = 0.5 * r["rho"] * r["V"] * r["V"] * 1.0
    force = (si["pressure_force"] - si["viscous_force"] * np.sqrt(1.4) * 0.1) * r["p"] * r["L"]
    assert abs(force[1] / dyn - golden["cl"]) <= 1e-12
    assert abs(force[0] / dyn - golden["cd"]) <= 5e-8
