"""Surface integrals of boundary zones on the device (the mesh functions behind the reference's lift,
drag, pressure and mass-flow monitors) against the oracle, whose integrals reproduce the
CylinderRe100 benchmark's lift and drag to 1e-12 (tests/test_oracle.py).

Cases: the reference cylinder mesh at uniform order with every zone kind; after a residual
evaluation of the resident state and after RK3 steps (the integrals then read the last stage's
input state, as the reference's monitors do).  FP64: each integral within 1e-12 of the zone's
pressure-integral scale; FP32 bulk: 1e-5.
"""
import numpy as np
import pytest

from oracle import oracle as O
import horses2d_b200 as hg
from cases_util import perturbed
from test_gpu_ns_parity import cylinder_ns

pytestmark = pytest.mark.gpu

KEYS = ("surface", "pressure", "pressure_force", "viscous_force", "mass_flow", "flow")


def compare(g, orc, tol):
    for zone in range(1, 6):
        a, b = g.surface_integrals(zone), orc.surface_integrals(zone)
        scale = abs(b["pressure"]) + abs(b["surface"]) + 1e-300
        for k in KEYS:
            np.testing.assert_allclose(a[k], b[k], rtol=0, atol=tol * scale, err_msg=f"zone {zone} {k}")


@pytest.mark.parametrize("viscous,ip", [(O.BR1, 0), (O.IP, 0)])
def test_cylinder_surface_integrals(viscous, ip):
    orc, kw, Q0 = cylinder_ns(4, O.LG, viscous, ip)
    Q = perturbed(Q0, 0.02, seed=41)
    orc.set_state(Q)
    orc.time_derivative(0.0)
    g = hg.GpuDGSEM(orc.export_mesh(), **kw)
    g.set_state(Q)
    g.compute_time_derivative(0.0)
    compare(g, orc, 1e-12)
    assert abs(orc.surface_integrals(5)["viscous_force"]).max() > 0.0
    dt = orc.estimate_dt(0.05, 1.0)
    for s in range(5):
        orc.time_step(O.RK3, s * dt, dt)
    g.time_steps(hg.SCHEME_RK3, 5, 0.0, dt)
    compare(g, orc, 1e-11)
    with pytest.raises(hg.HorsesGpuError):
        g.surface_integrals(6)


def test_cylinder_surface_integrals_fp32():
    orc, kw, Q0 = cylinder_ns(4, O.LG, O.BR1)
    Q = perturbed(Q0, 0.02, seed=42)
    orc.set_state(Q)
    orc.time_derivative(0.0)
    g = hg.GpuDGSEM(orc.export_mesh(), precision=hg.PREC_FP32, **kw)
    g.set_state(Q)
    g.compute_time_derivative(0.0)
    compare(g, orc, 1e-5)


def test_probes_match_oracle():
    """Probes (element + reference coordinates, located by mesh.locate on the cylinder O-grid) of the
    resident state: BilinearForm of the element's nodal values, against the oracle's, to 1e-13;
    a probe placed on a node returns the node's value."""
    from horses2d_b200 import mesh as hmesh
    orc, kw, Q0 = cylinder_ns(4, O.LG, O.BR1)
    Q = perturbed(Q0, 0.02, seed=43)
    orc.set_state(Q)
    desc = orc.export_mesh()
    g = hg.GpuDGSEM(desc, **kw)
    g.set_state(Q)
    pts = np.array([[0.75, 0.0], [0.6, 0.3], [-1.5, 0.7], [2.0, -1.0]])
    el, xe = hmesh.locate(desc, pts, hg.NODES_LG)
    xi, _ = hg.lib.nodes(4, hg.NODES_LG)
    el = np.append(el, 7)
    xe = np.vstack([xe, [xi[2], xi[3]]])
    out = g.probes(el, xe)
    for k in range(len(el)):
        np.testing.assert_allclose(out[k], orc.probe(el[k], xe[k, 0], xe[k, 1]), rtol=1e-13, atol=1e-13)
    np.testing.assert_array_equal(out[-1], Q.reshape(-1, 25, 4)[7, 3 * 5 + 2])
    with pytest.raises(hg.HorsesGpuError):
        g.probes([0], [[1.5, 0.5]])
