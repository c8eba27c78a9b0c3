"""Device health status of the stepped state (the reference's "The simulation has crashed",
Approximation/DGTimeIntegrator.f90:224-233): every RK update checks its nodes for a non-finite value,
rho <= 0 or p <= 0.  The bad states are made on the host (a NaN, a negative density, a negative pressure
written into the state before hg_set_state); nothing faults on the device."""
import numpy as np
import pytest

import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases

pytestmark = pytest.mark.gpu


def vortex(ns=False, precision=hg.PREC_FP64):
    d = hmesh.box_descriptor(8, 8, -5.0, 5.0, -5.0, 5.0, 4, hg.NODES_LGL)
    x = d["x"].reshape(-1, 2)
    Q = cases.isentropic_vortex(x[:, 0], x[:, 1], mach=0.5).ravel()
    kw = dict(mach=0.5, node_type=hg.NODES_LGL, riemann=hg.ROE, bcs=[dict(type=hg.BC_PERIODIC)] * 4)
    if ns:
        kw.update(navier_stokes=1, reynolds=200.0, viscous=hg.IP, ip_method=hg.SIPG, sigma0_ip=10.0)
    return hg.GpuDGSEM(d, precision=precision, **kw), Q


def poisoned(Q, kind, element=11, P=5):
    Q = Q.copy().reshape(-1, P * P, 4)
    if kind == "nan":
        Q[element, 7, 1] = np.nan
    elif kind == "density":
        Q[element, :, 0] = -0.5
    else:   # pressure: total energy below the kinetic energy
        Q[element, :, 3] = 0.01 * Q[element, :, 3]
    return Q.ravel()


@pytest.mark.parametrize("ns", [False, True])
def test_nan_fails_the_next_call_and_a_new_state_clears_it(ns):
    g, Q = vortex(ns)
    g.set_state(Q)
    g.time_step(hg.SCHEME_RK3, 0.0, 1e-3)
    assert g.health() == (0, -1)                       # a clean run stays clean
    g.set_state(poisoned(Q, "nan"))
    g.time_step(hg.SCHEME_RK3, 0.0, 1e-3)              # asynchronous: the step itself is queued
    bits, el = g.health()
    assert bits & hg.HEALTH_NONFINITE and 0 <= el < 64
    with pytest.raises(hg.HorsesGpuError) as ex:
        g.time_step(hg.SCHEME_RK3, 1e-3, 1e-3)
    assert ex.value.status == hg.STATUS_CRASHED and "crashed" in str(ex.value)
    with pytest.raises(hg.HorsesGpuError):
        g.residuals()
    g.set_state(Q)                                    # a new state clears the record
    assert g.health() == (0, -1)
    g.time_steps(hg.SCHEME_RK3, 6, 0.0, 1e-3)
    assert np.all(np.isfinite(g.residuals()))


@pytest.mark.parametrize("ns", [False, True])
@pytest.mark.parametrize("kind,bit", [("density", hg.HEALTH_DENSITY), ("pressure", hg.HEALTH_PRESSURE)])
def test_negative_density_and_pressure_are_recorded_and_fatal_on_request(ns, kind, bit):
    g, Q = vortex(ns)
    g.set_state(poisoned(Q, kind))
    g.time_step(hg.SCHEME_RK3, 0.0, 1e-3)
    bits, el = g.health()
    assert bits & (bit | hg.HEALTH_NONFINITE) and 0 <= el < 64
    if not bits & hg.HEALTH_NONFINITE:                 # recorded, not fatal under the default policy
        g.time_step(hg.SCHEME_RK3, 1e-3, 1e-3)
    g.set_health_policy(hg.HEALTH_NONFINITE | hg.HEALTH_DENSITY | hg.HEALTH_PRESSURE)
    with pytest.raises(hg.HorsesGpuError) as ex:
        g.time_step(hg.SCHEME_RK3, 2e-3, 1e-3)
    assert ex.value.status == hg.STATUS_CRASHED
    g.set_state(Q)
    g.time_steps(hg.SCHEME_RK3, 6, 0.0, 1e-3)         # clean under the strict policy
    assert g.health() == (0, -1)


def test_multi_step_call_and_fp32_path_report_it():
    g, Q = vortex(False, hg.PREC_FP32)
    g.set_state(poisoned(Q, "nan"))
    g.time_steps(hg.SCHEME_RK3, 8, 0.0, 1e-3)
    with pytest.raises(hg.HorsesGpuError) as ex:
        g.synchronize()
    assert ex.value.status == hg.STATUS_CRASHED
    assert g.health()[0] & hg.HEALTH_NONFINITE
