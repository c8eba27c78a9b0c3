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
