"""Restart files with a resident state: saving, reloading into a fresh context and continuing gives the
uninterrupted run bit for bit; the integration loop writes the reference's autosave files (every
`Autosave interval` iterations, named <solution>_<iter>.HiORst, and the final solution file)."""
import numpy as np
import pytest

import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases, restart

pytestmark = pytest.mark.gpu


def vortex(n=8, N=4, precision=hg.PREC_FP64):
    d = hmesh.box_descriptor(n, n, -5.0, 5.0, -5.0, 5.0, N, hg.NODES_LGL)
    x = d["x"].reshape(-1, 2)
    Q = cases.isentropic_vortex(x[:, 0], x[:, 1], beta=5.0, xc=0.0, yc=0.0).ravel()
    g = hg.GpuDGSEM(d, mach=0.5, node_type=hg.NODES_LGL, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4,
                    precision=precision)
    g.set_state(Q)
    return g


@pytest.mark.parametrize("precision", [hg.PREC_FP64, hg.PREC_FP32])
def test_save_load_continue_is_bitwise(tmp_path, precision):
    dt = 0.02
    a = vortex(precision=precision)
    a.time_steps(hg.SCHEME_RK3, 10, 0.0, dt)
    b = vortex(precision=precision)
    b.time_steps(hg.SCHEME_RK3, 5, 0.0, dt)
    p = tmp_path / "mid.HiORst"
    b.save_restart(p, 5 * dt, 5)
    t, it, Q = restart.read(p)
    assert (t, it) == (5 * dt, 5) and np.array_equal(Q, b.state())
    c = vortex(precision=precision)
    t, it = c.load_restart(p)
    assert (t, it) == (5 * dt, 5) and np.array_equal(c.state(), b.state())
    c.time_steps(hg.SCHEME_RK3, 5, t, dt)
    assert np.array_equal(c.state(), a.state())
    np.testing.assert_array_equal(c.residuals(), a.residuals())


def test_integrate_autosaves_and_restarts(tmp_path):
    sol = str(tmp_path / "Vortex.HiORst")
    kw = dict(transient=True, t_end=10.0, cfl=0.3, dt_cap=1.0, estimate_interval=100)
    a = vortex()
    it, t = a.integrate(hg.SCHEME_RK3, t0=0.0, max_iter=12, autosave_interval=4, solution_file=sol, **kw)
    assert it == 12
    for k in (4, 8, 12):
        assert (tmp_path / f"Vortex_{k}.HiORst").exists()
    tf, itf, Qf = restart.read(sol)
    assert (tf, itf) == (t, 12) and np.array_equal(Qf, a.state())
    t12, it12, Q12 = restart.read(tmp_path / "Vortex_12.HiORst")
    assert (t12, it12) == (t, 12) and np.array_equal(Q12, Qf)
    # the iteration-8 file is the state of a run stopped after 8 iterations
    b = vortex()
    it8, t8 = b.integrate(hg.SCHEME_RK3, t0=0.0, max_iter=8, **kw)
    c = vortex(n=8)
    tc, itc = c.load_restart(tmp_path / "Vortex_8.HiORst")
    assert (tc, itc) == (t8, 8) and np.array_equal(c.state(), b.state())


def test_load_restart_size_mismatch(tmp_path):
    a = vortex(n=4)
    p = tmp_path / "small.HiORst"
    a.save_restart(p, 0.0, 0)
    b = vortex(n=6)
    with pytest.raises(OSError, match="holds"):
        b.load_restart(p)


@pytest.mark.parametrize("mixed", [False, True])
def test_async_save_while_stepping(tmp_path, mixed):
    """hg_save_restart_async: the file holds the state of the requested iteration although steps are
    queued right after the call (single-order and mixed-order contexts)."""
    if mixed:
        d = hmesh.box_descriptor(5, 5, -5.0, 5.0, -5.0, 5.0, np.where(np.arange(25) % 5 % 2 == 1, 5, 3),
                                 hg.NODES_LG)
        x = d["x"].reshape(-1, 2)
        Q0 = cases.isentropic_vortex(x[:, 0], x[:, 1], beta=5.0).ravel()
        mk = lambda: hg.GpuDGSEM(d, mach=0.5, node_type=hg.NODES_LG, riemann=hg.ROE,  # noqa: E731
                                 bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    else:
        mk = vortex
    a = mk()
    if mixed:
        a.set_state(Q0)
    dt = 0.01
    a.time_steps(hg.SCHEME_RK3, 3, 0.0, dt)
    expect = a.state()
    a.save_restart(tmp_path / "async.HiORst", 3 * dt, 3, wait=False)
    a.time_steps(hg.SCHEME_RK3, 10, 3 * dt, dt)     # queued behind the copy
    a.restart_wait()
    t, it, Q = restart.read(tmp_path / "async.HiORst")
    assert (t, it) == (3 * dt, 3) and np.array_equal(Q, expect)
    a.save_restart(tmp_path / "sync.HiORst", 3 * dt, 3)
    assert not np.array_equal(restart.read(tmp_path / "sync.HiORst")[2], expect)   # the state moved on
    with pytest.raises(hg.HorsesGpuError, match="restart write"):
        a.save_restart(tmp_path / "no_such_dir" / "x.HiORst", 0.0, 0, wait=False)
        a.restart_wait()
