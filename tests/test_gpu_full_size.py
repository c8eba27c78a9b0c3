"""The C5 workload at its full size (1024 x 1024 periodic elements, N = 7, NDOF 268,435,456), where the
oracle cannot follow, checked through size-independent properties.

* FP64: on a periodic box the scheme is conservative (DGSpatialDiscretizationMethods.f90: every face flux
  enters its two elements with opposite signs; the interior-penalty and gradient-face terms integrate to
  zero against a constant), so over RK3 steps the quadrature integrals of rho, rho u, rho v and rho E move
  only by round-off.  Measured as |sum w dQ| / sum w |dQ| per variable, with dQ the change of the state
  at each node (Legendre-Gauss weights; the Jacobian is the same for every element of the uniform box):
  a flux that entered one side only would make the ratio of order one; round-off gives about 1e-9 here
  (over three steps a node changes by about 1e-9 while each update Q + c G rounds at ulp(Q) ~ 2e-16,
  and on the uniform part of the layer every element rounds the same way, so it adds up instead of
  averaging out; bound 1e-6).
* FP32 bulk: its time derivative of the initial state differs from the FP64 one by no more than the
  FP32 round-off floor of the same discretisation -- the FP32 time derivative of a uniform stream, which
  is zero in exact arithmetic (the volume and surface terms of a constant flux cancel, each of size
  |F| N^2 / h, so the floor is about 1e-7 of that: 1e-2 per node at h = 1/1024); its steps stay finite.
  At this size the floor is comparable to the time derivative of the shear layer itself, so a relative
  L2 against FP64 would be O(1) and says nothing; a wrong index or sign would sit far above the floor.
"""
import numpy as np
import pytest

import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh, cases

pytestmark = pytest.mark.gpu

N, NE = 7, 1024
DT = 0.05 / NE ** 2        # the workload's step (interior-penalty limited)
STEPS = 3


def kh_kwargs():
    return dict(mach=0.3, reynolds=1.0e4, navier_stokes=1, viscous=hg.IP, ip_method=hg.SIPG, sigma0_ip=10.0,
                node_type=hg.NODES_LG, riemann=hg.ROE, av_type=hg.AV_LAPLACIAN, av_intensity=1.0,
                bcs=[dict(type=hg.BC_PERIODIC)] * 4)


def conservation_ratios(Q0, Q1, w):
    ww = np.outer(w, w).reshape(-1)                       # node j*P+i
    d = (Q1 - Q0).reshape(-1, (N + 1) ** 2, 4)
    net = np.einsum("env,n->v", d, ww)
    tot = np.einsum("env,n->v", np.abs(d), ww)
    return np.abs(net) / tot, tot


def run(desc, Q0, precision):
    """(time derivative of Q0, state after STEPS RK3 steps)."""
    g = hg.GpuDGSEM(desc, precision=precision, **kh_kwargs())
    assert g.ndof == 4 * NE * NE * (N + 1) ** 2
    g.set_sensor(hg.SENSOR_MODAL)
    g.set_state(Q0)
    R = g.compute_time_derivative(0.0)
    g.set_state(Q0)
    g.time_steps(hg.SCHEME_RK3, STEPS, 0.0, DT)
    Q1 = g.state()
    g.close()
    assert np.all(np.isfinite(R)) and np.all(np.isfinite(Q1))
    return R, Q1


def test_kh_full_size_conservation_fp64_and_fp32_against_fp64():
    xi, w = np.polynomial.legendre.leggauss(N + 1)
    xi, w = 0.5 * (xi + 1.0), 0.5 * w
    desc = hmesh.box_descriptor(NE, NE, 0.0, 1.0, 0.0, 1.0, N, hg.NODES_LG)
    Q0 = cases.kelvin_helmholtz_box(NE, N, xi)
    R64, Q64 = run(desc, Q0, hg.PREC_FP64)
    r, tot = conservation_ratios(Q0, Q64, w)
    print(f"FP64: |sum w dQ| / sum w |dQ| per variable {r}, sum w |dQ| {tot}")
    assert np.all(tot > 0.0)           # the state moved
    assert np.all(r <= 1e-6)
    R32, _ = run(desc, Q0, hg.PREC_FP32)
    U = np.sqrt(1.4) * 0.3
    Qu = np.tile(np.array([1.0, U, 0.0, 1.0 / 0.4 + 0.5 * U * U]), NE * NE * (N + 1) ** 2)
    g = hg.GpuDGSEM(desc, precision=hg.PREC_FP32, **kh_kwargs())
    g.set_sensor(hg.SENSOR_MODAL)
    g.set_state(Qu)
    floor = float(np.linalg.norm(g.compute_time_derivative(0.0)))
    g.close()
    d = float(np.linalg.norm(R32 - R64))
    print(f"FP32 vs FP64 time derivative of the initial state: |R32 - R64| {d:.3e}, |R64| "
          f"{np.linalg.norm(R64):.3e}, FP32 floor (uniform stream) {floor:.3e}")
    assert floor > 0.0 and d <= 3.0 * floor
