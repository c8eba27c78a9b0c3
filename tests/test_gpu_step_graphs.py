"""Single-step CUDA graphs behind hg_time_step: stepping one call at a time (the reference's loop with
a residual check per iteration) replays a captured graph of one step per trace-buffer parity.  The
replays must give exactly the plain launches (bitwise), across parities (RK5 and Euler have an odd
number of stages), dt and scheme changes, and interleaved multi-step calls."""
import numpy as np
import pytest

import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases

pytestmark = pytest.mark.gpu


def ctx(ns=False, precision=hg.PREC_FP64, mixed=False):
    # mixed: a composite of two orders (a band of order 5; periodic partners share order 4)
    N = np.where(np.isin(np.arange(64) % 8, (3, 4)), 5, 4) if mixed else 4
    d = hmesh.box_descriptor(8, 8, -5.0, 5.0, -5.0, 5.0, N, hg.NODES_LG)
    x = d["x"].reshape(-1, 2)
    Q = cases.isentropic_vortex(x[:, 0], x[:, 1], beta=4.0).ravel()
    kw = dict(mach=0.5, node_type=hg.NODES_LG, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    if ns:
        kw.update(navier_stokes=1, reynolds=200.0, viscous=hg.BR1)
    g = hg.GpuDGSEM(d, precision=precision, **kw)
    g.set_state(Q)
    return g


@pytest.mark.parametrize("ns,mixed", [(False, False), (True, False), (False, True), (True, True)])
def test_single_step_graphs_equal_plain_launches(ns, mixed):
    a, b = ctx(ns, mixed=mixed), ctx(ns, mixed=mixed)
    b.profile(True)            # timing mode: plain launches only
    plan = [(hg.SCHEME_RK5, 0.01)] * 7 + [(hg.SCHEME_RK5, 0.008)] * 5 + [(hg.SCHEME_RK3, 0.008)] * 6 + \
           [(hg.SCHEME_EULER, 0.001)] * 5
    t = 0.0
    for k, (scheme, dt) in enumerate(plan):
        a.time_step(scheme, t, dt)
        b.time_step(scheme, t, dt)
        np.testing.assert_array_equal(a.residuals(), b.residuals())
        if k == 9:   # a multi-step call in between (pair graphs)
            a.time_steps(scheme, 6, t, dt)
            b.time_steps(scheme, 6, t, dt)
        t += dt
    assert np.array_equal(a.state(), b.state())
    # the surface traces of the last evaluation follow the replayed parity
    np.testing.assert_array_equal(a.compute_time_derivative(t), b.compute_time_derivative(t))


def test_boundary_states_between_steps_reach_the_replayed_graphs():
    """A Dirichlet zone fed per node (hg_set_boundary_state) with new states between single steps: the
    replayed step graphs read the zone's state buffer at replay time, so they give exactly what plain
    launches give with the same states (the first call for a zone grows that buffer and drops the
    captured graphs; later calls rewrite it in place).  Navier-Stokes on the reference cylinder mesh
    (viscous wall, far field, outlet), as in the per-node zone parity test."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from cases_util import perturbed
    from test_gpu_ns_parity import cylinder_ns
    from oracle import oracle as O
    orc, kw, Q0 = cylinder_ns(4, O.LG, O.BR1)
    Q = perturbed(Q0, 0.01, seed=12)
    Xb = orc.zone_edge_nodes(1)
    q = orc.zone_state(1)
    a, b = hg.GpuDGSEM(orc.export_mesh(), **kw), hg.GpuDGSEM(orc.export_mesh(), **kw)
    b.profile(True)            # timing mode: plain launches only
    for g in (a, b):
        g.set_state(Q)
    orc.set_state(Q)
    dt = orc.estimate_dt(0.2, 1.0)
    t = 0.0
    for k in range(12):
        if k in (0, 4, 5, 9):
            uB = (q[None, :] * (1.0 + 0.02 * np.sin((k + 2) * Xb[:, 0:1]))).ravel()
            a.set_boundary_state(1, uB)
            b.set_boundary_state(1, uB)
        a.time_step(hg.SCHEME_RK3, t, dt)
        b.time_step(hg.SCHEME_RK3, t, dt)
        np.testing.assert_array_equal(a.residuals(), b.residuals())
        t += dt
    sa, sb = a.state(), b.state()
    assert np.all(np.isfinite(sa)) and np.array_equal(sa, sb)
