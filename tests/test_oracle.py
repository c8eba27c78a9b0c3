"""The oracle against the reference's own golden vectors and known answers (CPU only).

* VortexTransport benchmark (TestCases/Benchmark/Simulations/VortexTransport):
  the reference's Finalize asserts iteration 3237 and the four max-norm errors
  w.r.t. the initial vortex to 1e-12 after integrating to t = 2 with Williamson
  RK5 (CFL 0.4, dt cap 1e-2) on a curved, p-refined (N = 5/7/12) mesh with
  mortars and periodic zones, Legendre-Gauss nodes and the Roe flux (the case
  file's "Inviscid Riemann Flux" key is not the one Setup.f90:280 reads, so the
  default Roe applies).
* Couette benchmark (TestCases/Benchmark/Simulations/Couette): Navier-Stokes
  with BR1, isothermal walls (one moving), a Dirichlet zone fed by the
  plugin's boundary-condition function and a partially non-reflective
  pressure outlet, on a p-refined (N = 5/7/10/7) curved mesh with mortars.
  The reference asserts iteration 19585 of the steady RK5 run (CFL 0.4,
  residual 1e-4) and the four final residuals to 1e-12.
* Ramp benchmark (TestCases/Benchmark/Simulations/Ramp): Navier-Stokes build at
  Re = 0 with IIPG, the jumps-based Laplacian artificial dissipation (intensity
  0.1), Euler walls and two newDirichlet zones, Mach 2, N = 3, Legendre-Gauss,
  steady RK5 (CFL 0.1, dt cap 2, residual 1e-8); the reference asserts
  iteration 9884 and the four final residuals to 1e-11.
* CylinderRe100 benchmark: exact Riemann solver on every zone, p-refinement, BR1, steady RK5; final
  residuals (1e-11) and the wall's lift and drag coefficients (surface integrals, 1e-12).
* CylinderRe1000 benchmark: SIPG interior penalty across p-refinement zones (orders 4-10), exact
  solver on every zone, transient RK5; iteration 512, residuals (1e-10), lift and drag (1e-12).
* Spectral building blocks: exactness of the nodal derivative and quadrature.
* Free-stream preservation on curved meshes, conservation on periodic meshes.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from cases_util import GOLDEN, load_mesh, vortex_case, rel_l2


def vortex_transport_ic(X, ref):
    """UserDefinedInitialCondition of the VortexTransport plugin, made dimensionless."""
    gamma, R, mach = 1.4, 287.15, 0.6
    cv, cp_d = R * 2.5, 3.5
    x, y = X[:, 0], X[:, 1]
    Rv, beta = 0.1, 0.05
    r2 = (x * x + y * y) / (Rv * Rv)
    u = ref["V"] * (np.cos(0.0) - beta * y / Rv * np.exp(-0.5 * r2))
    v = ref["V"] * (np.sin(0.0) + beta * x / Rv * np.exp(-0.5 * r2))
    T = ref["T"] * (1.0 - gamma * mach * mach * beta * beta / (2.0 * cp_d) * np.exp(-r2))
    rho = ref["rho"] * (T / ref["T"]) ** 2.5
    q = np.stack([rho, rho * u, rho * v, cv * (rho * T) + 0.5 * rho * (u * u + v * v)], 1)
    return q / np.array([ref["rho"], ref["rho"] * ref["a"], ref["rho"] * ref["a"], ref["p"]])


def vortex_transport_oracle():
    m = load_mesh("VortexTransportBench")
    porder = np.array([5, 7, 12, 7])[m["p_zones"]]
    bcs = [dict(type=O.BC_PERIODIC, periodic_dir=2, connected_marker=2),
           dict(type=O.BC_PERIODIC, periodic_dir=2, connected_marker=1),
           dict(type=O.BC_PERIODIC, periodic_dir=1, connected_marker=4),
           dict(type=O.BC_PERIODIC, periodic_dir=1, connected_marker=3)]
    return O.Oracle(m, porder, nodes=O.LG, riemann=O.ROE, mach=0.6, reynolds=0.0, bcs=bcs)


def test_vortex_transport_benchmark_golden():
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["VortexTransport"]
    orc = vortex_transport_oracle()
    # the mesh exercises every edge kind the benchmark relies on
    assert orc.edge_count(1) > 0 and orc.edge_count(2) > 0 and orc.edge_count(3) > 0
    X = orc.coords()
    orc.set_state(vortex_transport_ic(X, orc.ref).ravel())
    it, t = orc.integrate(O.RK5, transient=True, t0=0.0, t_end=2.0, max_iter=1000000, cfl=0.4, dt_cap=1e-2)
    err = np.abs(vortex_transport_ic(X, orc.ref) - orc.state().reshape(-1, 4)).max(0)
    assert it == golden["expected_iter"]
    assert np.max(np.abs(err - np.array(golden["expectedErrors"]))) <= 1e-12


@pytest.mark.parametrize("nodes", [O.LG, O.LGL])
def test_freestream_preservation_curved(nodes):
    """A uniform state has zero residual on the curved, p-refined reference mesh (metric identities)."""
    orc = vortex_transport_oracle() if nodes == O.LG else None
    if orc is None:
        m = load_mesh("VortexTransportBench")
        bcs = [dict(type=O.BC_PERIODIC, periodic_dir=2, connected_marker=2),
               dict(type=O.BC_PERIODIC, periodic_dir=2, connected_marker=1),
               dict(type=O.BC_PERIODIC, periodic_dir=1, connected_marker=4),
               dict(type=O.BC_PERIODIC, periodic_dir=1, connected_marker=3)]
        orc = O.Oracle(m, 4, nodes=nodes, riemann=O.ROE, mach=0.6, bcs=bcs)
    u = np.sqrt(1.4) * 0.6
    q = np.array([1.0, u, 0.0, 2.5 + 0.5 * u * u])
    orc.set_state(np.tile(q, orc.ndof // 4))
    qd = orc.time_derivative(0.0)
    # discrete metric identities hold to ~1e-9 on this mesh (curve degree NLow/2 on mortars)
    assert np.abs(qd).max() < 1e-8


def test_conservation_periodic():
    """On a periodic mesh the weighted sum of QDot (total mass, momentum, energy rate) vanishes."""
    orc, Q0, _ = vortex_case(n=8, N=4, nodes=O.LG)
    orc.set_state(Q0)
    qd = orc.time_derivative(0.0).reshape(orc.n_elements, -1, 4)
    Ja, jac, vol = orc.geometry()
    # Legendre-Gauss quadrature weights mapped to [0,1]
    x, w = np.polynomial.legendre.leggauss(5)
    W = np.outer(0.5 * w, 0.5 * w).ravel()     # (eta, xi) order matches node order j*P+i
    total = (qd * (jac.reshape(orc.n_elements, -1) * W)[:, :, None]).sum((0, 1))
    assert np.abs(total).max() < 1e-12 * np.abs(qd).max() * orc.n_elements


def test_rk3_matches_explicit_formula():
    """Williamson 2N RK3 in the oracle equals the three-stage update written out."""
    orc, Q0, _ = vortex_case(n=4, N=3)
    orc.set_state(Q0)
    dt = 1e-3
    orc.time_step(O.RK3, 0.0, dt)
    Q_rk = orc.state()
    orc.set_state(Q0)
    am, gm = [0.0, -5.0 / 9.0, -153.0 / 128.0], [1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0]
    Q, G = Q0.copy(), np.zeros_like(Q0)
    for m in range(3):
        orc.set_state(Q)
        k = orc.time_derivative(0.0)
        G = k if m == 0 else am[m] * G + k
        Q = Q + gm[m] * dt * G
    assert rel_l2(Q_rk, Q) < 1e-15


def couette_state(x, y, ref):
    """Couette profile of the Couette plugin's initial and boundary-condition functions (dimensional)."""
    R = 287.15
    cp, cv = R * 3.5, R * 2.5
    T = ref["T"] - ref["V"] ** 2 * 0.72 / (8.0 * cp) * (y + 1.0) * (y - 1.0)
    rho = 101325.0 / (R * T)
    rhou = rho * ref["V"] * 0.5 * (y + 1.0)
    return np.stack([rho, rhou, 0.0 * y, cv * rho * T + 0.5 * rhou * rhou / rho], 1)


def test_couette_benchmark_golden():
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["Couette"]
    m = load_mesh("CouetteBench")
    porder = np.array([5, 7, 10, 7])[m["p_zones"]]
    bcs = [dict(type=O.BC_VISCOUSWALL, wall_type=1),
           dict(type=O.BC_VISCOUSWALL, wall_type=1, wall_v=(np.sqrt(1.4) * 0.8, 0.0)),
           dict(type=O.BC_DIRICHLET),
           dict(type=O.BC_PRESSUREOUTLET, outflow_type=2)]
    orc = O.Oracle(m, porder, nodes=O.LG, riemann=O.ROE, mach=0.8, reynolds=2000.0, prandtl=0.72,
                   navier_stokes=1, viscous=O.BR1, bcs=bcs)
    ref = orc.ref
    scale = np.array([ref["rho"], ref["rho"] * ref["a"], ref["rho"] * ref["a"], ref["p"]])
    X = orc.coords()
    q0 = couette_state(X[:, 0], X[:, 1], ref)
    q0[X[:, 0] ** 2 + X[:, 1] ** 2 < 0.005, 1] *= 1.005
    orc.set_state((q0 / scale).ravel())
    Xb = orc.zone_edge_nodes(3)
    orc.set_zone_state(3, (couette_state(Xb[:, 0], Xb[:, 1], ref) / scale).ravel())
    it, _ = orc.integrate(O.RK5, transient=False, t0=0.0, t_end=1.0, max_iter=100000, cfl=0.4, dt_cap=1.0,
                          residual_target=1e-4)
    assert it == golden["expected_iter"]
    assert np.max(np.abs(orc.residuals() - np.array(golden["expectedResiduals"]))) <= 1e-12


def test_ns_freestream_preservation_curved():
    """Uniform flow is a discrete steady state of the NS residual on curved meshes (BR1 and IP)."""
    m = load_mesh("CylinderBench")
    for viscous in (O.BR1, O.IP):
        orc = O.Oracle(m, 4, nodes=O.LG, riemann=O.ROE, mach=0.3, reynolds=100.0, navier_stokes=1, viscous=viscous,
                       bcs=[dict(type=O.BC_DIRICHLET)] * 5)
        q = np.array([1.0, 0.3 * np.sqrt(1.4), 0.0, 2.5 + 0.5 * 0.09 * 1.4])
        orc.set_state(np.tile(q, orc.ndof // 4))
        assert np.abs(orc.time_derivative(0.0)).max() <= 1e-8


def test_cylinder_re100_benchmark_golden():
    """CylinderRe100 (TestCases/Benchmark/Simulations/CylinderRe100): Navier-Stokes, Re 100, M 0.1, BR1,
    HLL inside and the exact Riemann solver on every zone (three Dirichlet zones, a partially
    non-reflective pressure outlet, an adiabatic wall), p-refinement zones of orders 2/8/6/4 on
    Legendre-Gauss nodes (mortars of the projection types 3-6), steady RK5 for 250 iterations at
    CFL 0.1, dt cap 1e-2.  The reference asserts the final residuals to 1e-11 and the lift and drag
    coefficients of the wall -- surface integrals of pressure and of the viscous tensor over the
    last stage's traces (Monitors.f90:1130-1138) -- to 1e-12."""
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["CylinderRe100"]
    m = load_mesh("CylinderBench")
    porder = np.array([8, 2, 8, 6, 4])[m["p_zones"]]     # zone 0 would take the default order 8
    ex = O.EXACT
    bcs = [dict(type=O.BC_DIRICHLET, riemann=ex), dict(type=O.BC_DIRICHLET, riemann=ex),
           dict(type=O.BC_DIRICHLET, riemann=ex), dict(type=O.BC_PRESSUREOUTLET, outflow_type=2, riemann=ex),
           dict(type=O.BC_VISCOUSWALL, wall_type=2, riemann=ex)]
    orc = O.Oracle(m, porder, nodes=O.LG, riemann=O.HLL, mach=0.1, reynolds=100.0, prandtl=0.72, navier_stokes=1,
                   viscous=O.BR1, bcs=bcs)
    r = orc.ref
    cv = 287.15 * 2.5   # UniformInitialCondition, dimensional
    q = np.array([r["rho"], r["rho"] * r["V"], 0.0, cv * r["rho"] * r["T"] + 0.5 * r["rho"] * r["V"] * r["V"]])
    q = q / np.array([r["rho"], r["rho"] * r["a"], r["rho"] * r["a"], r["p"]])
    orc.set_state(np.tile(q, orc.ndof // 4))
    it, _ = orc.integrate(O.RK5, transient=False, t0=0.0, t_end=1e9, max_iter=250, cfl=0.1, dt_cap=1e-2,
                          residual_target=1e-14)
    assert it == 250
    assert np.max(np.abs(orc.residuals() - np.array(golden["residuals"]))) <= 1e-11
    # lift / drag surface monitors: (pressure force - sqrt(gamma) M viscous force) p_ref L / (rho V^2 S / 2)
    si = orc.surface_integrals(5)
    dyn = 0.5 * r["rho"] * r["V"] * r["V"] * 1.0
    force = (si["pressure_force"] - si["viscous_force"] * np.sqrt(1.4) * 0.1) * r["p"] * r["L"]
    assert abs(force[1] / dyn - golden["cl"]) <= 1e-12
    assert abs(force[0] / dyn - golden["cd"]) <= 1e-12


def cylinder_re1000_oracle(ip_method=0):
    """CylinderRe1000 (TestCases/Benchmark/Simulations/CylinderRe1000): Navier-Stokes, Re 1000, M 0.1,
    SIPG interior penalty (sigma0 10), HLL inside and the exact solver on every zone (three Dirichlet
    zones, a partially non-reflective pressure outlet, an adiabatic wall), p-refinement zones of
    orders 6/10/8/8 around the default 4, Legendre-Gauss nodes, uniform initial state."""
    m = load_mesh("CylinderInflation")
    porder = np.array([4, 6, 10, 8, 8])[m["p_zones"]]
    ex = O.EXACT
    bcs = [dict(type=O.BC_DIRICHLET, riemann=ex), dict(type=O.BC_DIRICHLET, riemann=ex),
           dict(type=O.BC_DIRICHLET, riemann=ex), dict(type=O.BC_PRESSUREOUTLET, outflow_type=2, riemann=ex),
           dict(type=O.BC_VISCOUSWALL, wall_type=2, riemann=ex)]
    orc = O.Oracle(m, porder, nodes=O.LG, riemann=O.HLL, mach=0.1, reynolds=1000.0, prandtl=0.72, navier_stokes=1,
                   viscous=O.IP, ip_method=ip_method, sigma0_ip=10.0, bcs=bcs)
    r = orc.ref
    cv = 287.15 * 2.5   # UniformInitialCondition, dimensional
    q = np.array([r["rho"], r["rho"] * r["V"], 0.0, cv * r["rho"] * r["T"] + 0.5 * r["rho"] * r["V"] * r["V"]])
    q = q / np.array([r["rho"], r["rho"] * r["a"], r["rho"] * r["a"], r["p"]])
    return orc, q


def test_cylinder_re1000_benchmark_golden():
    """The reference asserts, after the transient RK5 run to t = 0.013 (CFL 0.1, dt cap 1e-2),
    iteration 512, the final residuals to 1e-10 and the wall's lift and drag to 1e-12
    (SETUP/ProblemFile.f90:79-95).  Pins interior penalty across p-nonconforming edges (projection
    types 3-6 of the viscous and gradient-face terms, penalty at the edge's order)."""
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["CylinderRe1000"]
    orc, q = cylinder_re1000_oracle()
    orc.set_state(np.tile(q, orc.ndof // 4))
    it, t = orc.integrate(O.RK5, transient=True, t0=0.0, t_end=0.013, max_iter=10000000, cfl=0.1, dt_cap=1e-2)
    assert it == golden["expected_iter"]
    assert np.max(np.abs(orc.residuals() - np.array(golden["residuals"]))) <= 1e-10
    r = orc.ref
    si = orc.surface_integrals(5)
    dyn = 0.5 * r["rho"] * r["V"] * r["V"] * 1.0
    force = (si["pressure_force"] - si["viscous_force"] * np.sqrt(1.4) * 0.1) * r["p"] * r["L"]
    assert abs(force[1] / dyn - golden["cl"]) <= 1e-12
    assert abs(force[0] / dyn - golden["cd"]) <= 1e-12


def test_ramp_benchmark_golden():
    golden = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["Ramp"]
    bcs = [dict(type=O.BC_EULERWALL), dict(type=O.BC_EULERWALL), dict(type=O.BC_NEWDIRICHLET),
           dict(type=O.BC_NEWDIRICHLET)]
    orc = O.Oracle(load_mesh("RampBench"), 3, nodes=O.LG, riemann=O.ROE, mach=2.0, reynolds=0.0, prandtl=0.72,
                   navier_stokes=1, viscous=O.IP, ip_method=2, sigma0_ip=1.0, bcs=bcs, av_type=O.AV_LAPLACIAN,
                   av_intensity=0.1)
    r = orc.ref
    cv = 287.15 * 2.5   # UniformInitialCondition (Generic/InitialConditions.f90:154-170), dimensional
    q = np.array([r["rho"], r["rho"] * r["V"], r["rho"] * r["V"] * np.sin(0.0),
                  cv * r["rho"] * r["T"] + 0.5 * r["rho"] * r["V"] * r["V"]])
    q = q / np.array([r["rho"], r["rho"] * r["a"], r["rho"] * r["a"], r["p"]])
    orc.set_state(np.tile(q, orc.ndof // 4))
    it, _ = orc.integrate(O.RK5, transient=False, t0=0.0, t_end=1.0, max_iter=20000, cfl=0.1, dt_cap=2.0,
                          residual_target=1e-8)
    assert it == golden["expected_iter"]
    assert np.max(np.abs(orc.residuals() - np.array(golden["residuals"]))) <= 1e-11


def test_cylinder_mach2_oracle_run_meets_the_reference_check():
    """CylinderMach2 (TestCases/Benchmark/Simulations/CylinderMach2/SETUP/ProblemFile.f90:79-95): the committed
    oracle run (tests/golden/make_cylinder_mach2_oracle.py, about 13 minutes on 8 threads) passes the
    reference's own assertions -- final iteration 15599, residuals to 1e-9, lift and drag to 1e-12.  The
    iteration count hinges on the dt estimate's MAX / MIN with the NaN sound speed of transient negative-
    pressure nodes (oracle/api.cpp run_max / run_min); NaN-ignoring maxima give 16079 steps."""
    import json
    ref = json.load(open(os.path.join(GOLDEN, "benchmarks.json")))["CylinderMach2"]
    run = json.load(open(os.path.join(GOLDEN, "cylinder_mach2_oracle.json")))
    assert run["iterations"] == ref["expected_iter"] == 15599 and run["t"] == 10.0
    assert np.max(np.abs(np.array(run["residuals"]) - np.array(ref["residuals"]))) <= 1e-9
    assert abs(run["cl"] - ref["cl"]) <= 1e-12 and abs(run["cd"] - ref["cd"]) <= 1e-12
