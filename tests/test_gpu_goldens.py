"""A reference benchmark run end to end on the device: CylinderMach2
(TestCases/Benchmark/Simulations/CylinderMach2) -- the cylinder mesh at N = 5, Legendre-Gauss, Roe,
Re = 0 with IIPG and the jumps-based Laplacian dissipation (intensity 0.4), Euler walls, a Dirichlet
inflow, a partially non-reflective pressure outlet, transient Williamson RK5 to t = 10 at CFL 0.05
(dt cap 1e-2, re-estimated every 100 iterations), built with the package's own mesh builder and driven
by GpuDGSEM.integrate (the reference's integration loop).

* Against the reference's own benchmark check (ProblemFile.f90:79-95, tests/golden/benchmarks.json):
  the final iteration 15599, residuals to 1e-9 and lift and drag to 1e-12, as the reference asserts.
  The iteration count depends on how the dt estimate's running maxima treat the NaN sound speed of
  nodes whose internal energy turns negative in the transient (hg_estimate_dt follows the reference's
  compiled MAX / MIN; with NaN-ignoring maxima the run takes 16079 steps).
* Against the oracle's run of the same setup (tests/golden/cylinder_mach2_oracle.json, written by
  make_cylinder_mach2_oracle.py): the same iterations, residuals to 1e-10 relative, lift and drag to
  1e-12 -- after 78,000 residual evaluations through a forming bow shock.
"""
import json
import os

import numpy as np
import pytest

import horses2d_b200 as hg
from horses2d_b200 import mesh as hmesh
from cases_util import GOLDEN, load_mesh

pytestmark = pytest.mark.gpu


def test_cylinder_mach2_benchmark_on_device():
    import torch
    ref = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["CylinderMach2"]
    orc = json.load(open(os.path.join(GOLDEN, "cylinder_mach2_oracle.json")))
    mach, N = 2.0, 5
    desc = hmesh.build_descriptor(load_mesh("CylinderBench"), N, hg.NODES_LG)
    u = np.sqrt(1.4) * mach
    q = np.array([1.0, u, 0.0, 2.5 + 0.5 * u * u])      # uniform initial condition, dimensionless
    g = hg.GpuDGSEM(desc, mach=mach, reynolds=0.0, prandtl=0.72, navier_stokes=1, viscous=hg.IP,
                    ip_method=hg.IIPG, sigma0_ip=1.0, node_type=hg.NODES_LG, riemann=hg.ROE,
                    av_type=hg.AV_LAPLACIAN, av_intensity=0.4,
                    bcs=[dict(type=hg.BC_EULERWALL), dict(type=hg.BC_EULERWALL), dict(type=hg.BC_DIRICHLET, state=q),
                         dict(type=hg.BC_PRESSUREOUTLET, state=q, outflow_type=2), dict(type=hg.BC_EULERWALL)])
    stream = torch.cuda.Stream()
    g.set_stream(stream.cuda_stream)
    g.set_state(np.tile(q, g.ndof // 4))
    it, t = g.integrate(hg.SCHEME_RK5, transient=True, t0=0.0, t_end=10.0, max_iter=200000, cfl=0.05, dt_cap=1e-2)
    assert t == 10.0
    res = g.residuals()
    si = g.surface_integrals(5)
    rho, V, p_ref = 101325.0 / (287.15 * 273.15), mach * np.sqrt(1.4 * 287.15 * 273.15), 101325.0
    force = si["pressure_force"] * p_ref / (0.5 * rho * V * V)     # Re = 0: no viscous force
    cl, cd = force[1], force[0]
    # the reference's benchmark check
    assert it == ref["expected_iter"] == 15599
    assert np.max(np.abs(res - np.array(ref["residuals"]))) <= 1e-9
    assert abs(cl - ref["cl"]) <= 1e-12
    assert abs(cd - ref["cd"]) <= 1e-12
    # the oracle's run
    assert it == orc["iterations"]
    np.testing.assert_allclose(res, orc["residuals"], rtol=1e-10, atol=0)
    assert abs(cl - orc["cl"]) <= 1e-12 and abs(cd - orc["cd"]) <= 1e-12
