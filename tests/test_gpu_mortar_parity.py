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
