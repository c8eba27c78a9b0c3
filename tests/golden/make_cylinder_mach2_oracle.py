"""Writes cylinder_mach2_oracle.json: the oracle's run of the CylinderMach2 benchmark setup
(TestCases/Benchmark/Simulations/CylinderMach2: the CylinderRe100 mesh at N = 5, Legendre-Gauss, Roe,
Re = 0 with IIPG and the jumps-based Laplacian dissipation (intensity 0.4), Euler walls, a Dirichlet
inflow, a partially non-reflective pressure outlet, transient Williamson RK5 to t = 10 at CFL 0.05,
dt cap 1e-2).  The GPU test replays the run on the device and compares with these values.
Takes about 8 minutes on 8 threads:  python tests/golden/make_cylinder_mach2_oracle.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O          # noqa: E402
from cases_util import load_mesh         # noqa: E402


def main():
    m = load_mesh("CylinderBench")
    bcs = [dict(type=O.BC_EULERWALL), dict(type=O.BC_EULERWALL), dict(type=O.BC_DIRICHLET),
           dict(type=O.BC_PRESSUREOUTLET, outflow_type=2), dict(type=O.BC_EULERWALL)]
    O.lib().or_set_threads(os.cpu_count() or 1)
    orc = O.Oracle(m, 5, nodes=O.LG, riemann=O.ROE, mach=2.0, reynolds=0.0, prandtl=0.72, navier_stokes=1,
                   viscous=O.IP, ip_method=2, sigma0_ip=1.0, bcs=bcs, av_type=O.AV_LAPLACIAN, av_intensity=0.4)
    r = orc.ref
    cv = 287.15 * 2.5
    q = np.array([r["rho"], r["rho"] * r["V"], 0.0, cv * r["rho"] * r["T"] + 0.5 * r["rho"] * r["V"] * r["V"]])
    q = q / np.array([r["rho"], r["rho"] * r["a"], r["rho"] * r["a"], r["p"]])
    orc.set_state(np.tile(q, orc.ndof // 4))
    it, t = orc.integrate(O.RK5, transient=True, t0=0.0, t_end=10.0, max_iter=200000, cfl=0.05, dt_cap=1e-2)
    si = orc.surface_integrals(5)
    dyn = 0.5 * r["rho"] * r["V"] * r["V"]
    F = si["pressure_force"] * r["p"] * r["L"]
    out = dict(iterations=it, t=t, residuals=orc.residuals().tolist(), cl=F[1] / dyn, cd=F[0] / dyn)
    with open(os.path.join(HERE, "cylinder_mach2_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
