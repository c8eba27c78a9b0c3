"""Context groups: an ensemble packed into one context per polynomial order, advanced by one CUDA
graph whose members run on forked streams.  The group must give exactly the members' own stepping
(same kernels, same order per member: bitwise equal), rebuild its graph when dt or a member's set-up
changes, and refuse members on different streams."""
import numpy as np
import pytest

from oracle import oracle as O
import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases
from cases_util import rel_l2

pytestmark = pytest.mark.gpu


def member(n, N, nodes, xc, beta, stream, precision=hg.PREC_FP64):
    d = hmesh.box_descriptor(n, n, -5.0, 5.0, -5.0, 5.0, N, nodes)
    x = d["x"].reshape(-1, 2)
    Q = cases.isentropic_vortex(x[:, 0], x[:, 1], beta=beta, xc=xc, yc=-xc).ravel()
    g = hg.GpuDGSEM(d, mach=0.5, node_type=nodes, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4,
                    precision=precision)
    g.set_stream(stream.cuda_stream)
    g.set_state(Q)
    return g, Q


def test_group_equals_members_stepped_alone():
    import torch
    s = torch.cuda.Stream()
    spec = [(6, 3, hg.NODES_LGL, 0.5, 4.0), (10, 5, hg.NODES_LG, -1.0, 5.0), (8, 7, hg.NODES_LGL, 1.5, 3.0)]
    grp_m = [member(*a, s) for a in spec]
    solo_m = [member(*a, s) for a in spec]
    grp = hg.GpuGroup([g for g, _ in grp_m])
    dt = 0.01
    grp.time_steps(hg.SCHEME_RK3, 7, 0.0, dt)      # 1 + 3 graph launches of 2 steps
    for g, _ in solo_m:
        g.time_steps(hg.SCHEME_RK3, 7, 0.0, dt)
    for (a, _), (b, _) in zip(grp_m, solo_m):
        assert np.array_equal(a.state(), b.state())
        np.testing.assert_array_equal(a.residuals(), b.residuals())
    # a new dt and a member's tiling change rebuild the graph; results stay equal
    grp_m[1][0].set_tiling(1)
    solo_m[1][0].set_tiling(1)
    grp.time_steps(hg.SCHEME_RK3, 4, 7 * dt, 0.5 * dt)
    for g, _ in solo_m:
        g.time_steps(hg.SCHEME_RK3, 4, 7 * dt, 0.5 * dt)
    for (a, _), (b, _) in zip(grp_m, solo_m):
        assert np.array_equal(a.state(), b.state())
    grp.close()


def test_group_member_against_oracle():
    import torch
    s = torch.cuda.Stream()
    g1, Q1 = member(8, 4, hg.NODES_LGL, 0.0, 5.0, s)
    g2, _ = member(6, 6, hg.NODES_LG, 1.0, 3.0, s)
    grp = hg.GpuGroup([g1, g2])
    orc = O.Oracle(hmesh.cartesian(8, 8, -5.0, 5.0, -5.0, 5.0), 4, nodes=O.LGL, riemann=O.ROE, mach=0.5,
                   bcs=hmesh.periodic_bcs_cartesian())
    orc.set_state(Q1)
    dt = orc.estimate_dt(0.4, 1.0)
    for k in range(10):
        orc.time_step(O.RK3, k * dt, dt)
    grp.time_steps(hg.SCHEME_RK3, 10, 0.0, dt)
    assert rel_l2(g1.state(), orc.state()) <= 1e-11
    grp.close()


def test_group_rejects_members_on_different_streams():
    import torch
    g1, _ = member(4, 3, hg.NODES_LGL, 0.0, 5.0, torch.cuda.Stream())
    g2, _ = member(4, 3, hg.NODES_LGL, 0.0, 5.0, torch.cuda.Stream())
    with pytest.raises(hg.HorsesGpuError):
        hg.GpuGroup([g1, g2])
    with pytest.raises(hg.HorsesGpuError):
        hg.GpuGroup([g1, g1])
