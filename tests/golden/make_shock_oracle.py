"""Writes shock_c3_oracle.npz: the oracle's density after 200 Williamson RK3 steps of the supersonic shock
workload at its full size (512 x 64 elements on [0,10] x [0,1], N = 3, Legendre-Gauss, HLL, Navier-Stokes
build at Re = 0 with SIPG, Laplacian artificial dissipation driven by the modal-decay indicator; a Mach-3
normal shock on the element face nearest x = 5 with an upstream entropy wave of amplitude 0.2; dt from the
reference's estimate at CFL 0.1).  The FP32-bulk device path is checked against it after the same 200 steps
(tests/test_gpu_config_parity.py).  The density is stored in float32 (relative precision 6e-8, far below the
1e-5 tolerance it serves).  About 2 minutes on 8 threads:  python tests/golden/make_shock_oracle.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O          # noqa: E402
from horses2d_b200 import mesh as hmesh, sensor as S   # noqa: E402

NX, NY, N, STEPS = 512, 64, 3, 200


def shock_oracle(indicator=O.IND_MODAL, nx=NX, ny=NY):
    """The shock workload's oracle and initial state (the sensor module's case on the oracle's mesh)."""
    (r1, u1, p1), (r2, u2, p2) = S.rankine_hugoniot(3.0)
    bcs = [dict(type=O.BC_EULERWALL), dict(type=O.BC_EULERWALL), dict(type=O.BC_DIRICHLET),
           dict(type=O.BC_NEWDIRICHLET, pressure=101325.0 * p2, temperature=273.15 * p2 / r2,
                mach=u2 / np.sqrt(1.4 * p2 / r2))]
    orc = O.Oracle(hmesh.cartesian(nx, ny, 0.0, 10.0, 0.0, 1.0), N, nodes=O.LG, riemann=O.HLL, mach=3.0,
                   reynolds=0.0, navier_stokes=1, viscous=O.IP, ip_method=0, sigma0_ip=10.0, bcs=bcs,
                   av_type=O.AV_LAPLACIAN, av_intensity=1.0, av_indicator=indicator)
    Q0 = S.shock_state({"x": orc.coords().ravel()}, S.snap_to_face(5.0, nx), 0.2).ravel()
    return orc, Q0


def main():
    O.lib().or_set_threads(os.cpu_count() or 1)
    orc, Q0 = shock_oracle()
    orc.set_state(Q0)
    dt = orc.estimate_dt(0.1, 1.0)
    for s in range(STEPS):
        orc.time_step(O.RK3, s * dt, dt)
    rho = orc.state()[0::4]
    assert np.all(np.isfinite(rho))
    np.savez_compressed(os.path.join(HERE, "shock_c3_oracle.npz"), rho=rho.astype(np.float32), dt=np.array([dt]),
                        steps=np.array([STEPS]))
    print("dt", dt, "rho range", rho.min(), rho.max())


if __name__ == "__main__":
    main()
