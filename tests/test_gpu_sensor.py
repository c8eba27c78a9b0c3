"""Shock sensors on the GPU: modal-decay indicator, learned (MLP) indicator and its training kernels.

* network kernels (forward, loss gradient) against the FP64 CPU restatement oracle/mlp.py
  (FP32 kernels: relative tolerance 1e-4 on the loss and the gradient);
* modal features and indicator against oracle/mlp.py (FP64 path);
* full residual with modal / learned artificial viscosity against the C++ oracle (FP64, 1e-12): the
  oracle's own modal indicator, and for the learned one the oracle fed the library's per-element G;
* out-of-distribution fallback to the modal indicator;
* GPU training decreases the loss.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import mlp as omlp
import horses2d_b200 as hg
from horses2d_b200 import sensor as S, mesh as hmesh
from cases_util import rel_l2

pytestmark = pytest.mark.gpu


def random_problem(n, seed):
    rng = np.random.default_rng(seed)
    p = (0.4 * rng.standard_normal(omlp.N_PARAMS)).astype(np.float32)
    X = rng.standard_normal((n, 16)).astype(np.float32)
    t = (rng.random(n) > 0.4).astype(np.float32)
    w = (0.5 + rng.random(n)).astype(np.float32)
    return p, X, t, w


def test_mlp_forward_and_gradient_match_oracle():
    p, X, t, w = random_problem(3000, 1)
    y = S.mlp_forward(p, X)
    np.testing.assert_allclose(y, omlp.predict(p, X), rtol=0, atol=2e-6)
    loss, g = S.mlp_grad(p, X, t, w)
    lref, gref = omlp.loss_grad(p, X, t, w)
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    assert np.max(np.abs(g - gref)) <= 1e-4 * np.max(np.abs(gref))
    # unit weights path
    loss1, g1 = S.mlp_grad(p, X, t)
    l1ref, g1ref = omlp.loss_grad(p, X, t)
    assert abs(loss1 - l1ref) <= 1e-5 * abs(l1ref)
    assert np.max(np.abs(g1 - g1ref)) <= 1e-4 * np.max(np.abs(g1ref))


def test_training_decreases_loss():
    rng = np.random.default_rng(2)
    X = rng.standard_normal((20000, 16)).astype(np.float32)
    t = (X[:, 0] + 0.5 * X[:, 3] - 0.3 * X[:, 7] > 0.2).astype(np.float32)
    params, hist = S.train(X, t, epochs=8, batch=1024, lr=3e-3, seed=3)
    assert hist[-1] < 0.3 * hist[0]
    acc = np.mean((S.mlp_forward(params, X) > 0.5) == (t > 0.5))
    assert acc > 0.95


def small_shock(nx=48, ny=4, N=3, precision=hg.PREC_FP64, indicator=O.IND_MODAL, sensor=hg.SENSOR_MODAL):
    """Oracle and GPU context of the shock / entropy-wave case at a small size (same state)."""
    m = hmesh.cartesian(nx, ny, 0.0, 10.0, 0.0, 1.0)
    (r1, u1, p1), (r2, u2, p2) = S.rankine_hugoniot(3.0)
    bcs = [dict(type=O.BC_EULERWALL), dict(type=O.BC_EULERWALL), dict(type=O.BC_DIRICHLET),
           dict(type=O.BC_NEWDIRICHLET, pressure=101325.0 * p2, temperature=273.15 * p2 / r2,
                mach=u2 / np.sqrt(1.4 * p2 / r2))]
    orc = O.Oracle(m, N, nodes=O.LG, riemann=O.HLL, mach=3.0, reynolds=0.0, navier_stokes=1, viscous=O.IP,
                   ip_method=0, sigma0_ip=10.0, bcs=bcs, av_type=O.AV_LAPLACIAN, av_intensity=1.0,
                   av_indicator=indicator)
    qin, qout = orc.zone_state(3), orc.zone_state(4)
    kw = dict(mach=3.0, reynolds=0.0, navier_stokes=1, viscous=hg.IP, ip_method=hg.SIPG, sigma0_ip=10.0,
              node_type=hg.NODES_LG, riemann=hg.HLL, av_type=hg.AV_LAPLACIAN, av_intensity=1.0,
              bcs=[dict(type=hg.BC_EULERWALL), dict(type=hg.BC_EULERWALL), dict(type=hg.BC_DIRICHLET, state=qin),
                   dict(type=hg.BC_NEWDIRICHLET, state=qout)])
    g = hg.GpuDGSEM(orc.export_mesh(), precision=precision, **kw)
    if sensor != hg.SENSOR_LEARNED:
        g.set_sensor(sensor)
    X = orc.coords()
    x = X[:, 0]
    up = x < 5.05
    Q = S.conservative(np.where(up, 1.0 + 0.2 * np.sin(5.0 * x), r2), np.where(up, u1, u2), np.where(up, 1.0, p2))
    Q = Q.ravel() * (1.0 + 1e-3 * np.random.default_rng(4).standard_normal(Q.size))
    return orc, g, Q


def test_modal_features_and_indicator_match_oracle():
    orc, g, Q = small_shock()
    g.set_state(Q)
    feats, out = g.sensor_eval()
    xi, _ = hg.lib.nodes(3, hg.NODES_LG)
    fref, sref = omlp.element_features(Q.reshape(-1, 16, 4), xi)
    np.testing.assert_allclose(feats, fref, rtol=0, atol=1e-5)
    gref = omlp.ramp(sref, np.log10(1.0 / 4 ** 4), 1.0)
    np.testing.assert_allclose(out[:, 0], gref, rtol=0, atol=1e-12)
    assert np.sum(out[:, 0] > 0.5) >= 4          # the shock column is flagged
    assert np.all(out[:, 1] == -1.0)              # no weights yet


def test_modal_artificial_viscosity_residual_parity():
    orc, g, Q = small_shock()
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    g.set_state(Q)
    out = g.compute_time_derivative(0.0)
    assert rel_l2(out, ref) <= 1e-12
    np.testing.assert_allclose(g.element_viscosity(), orc.av_viscosity(), rtol=1e-12, atol=1e-300)
    assert np.max(orc.av_viscosity()) > 0.0


def test_learned_sensor_residual_parity_and_fallback():
    orc, g, Q = small_shock(indicator=O.IND_EXTERNAL, sensor=hg.SENSOR_LEARNED)
    p, _, _, _ = random_problem(1, 7)
    g.set_state(Q)
    feats, _ = g.sensor_eval()
    lo, hi = S.feature_box(feats[: len(feats) // 2], margin=0.0, pad=0.0)   # leaves some elements outside
    g.set_sensor(hg.SENSOR_LEARNED, mlp=p, lo=lo, hi=hi)
    _, out = g.sensor_eval()
    ood = out[:, 2] > 0.5
    assert 0 < ood.sum() < len(ood)
    np.testing.assert_array_equal(out[ood, 3], out[ood, 0])        # fallback: modal G
    np.testing.assert_allclose(out[~ood, 3], out[~ood, 1], rtol=0, atol=0)
    np.testing.assert_allclose(out[:, 1], omlp.learned_g(S.mlp_forward(p, feats)), rtol=0, atol=1e-6)
    orc.set_av_g(out[:, 3])
    orc.set_state(Q)
    ref = orc.time_derivative(0.0)
    res = g.compute_time_derivative(0.0)
    assert rel_l2(res, ref) <= 1e-12


def test_learned_sensor_end_to_end_gain_over_modal():
    """Train on plain-solver snapshots (two rounds), then run held-out shock cases with each indicator
    driving the artificial viscosity.  The learned indicator finds the whole shock band (the modal one,
    at its default calibration, flags only the element holding the jump) with few false positives, and
    the standing shock of the solution moves no further from where it started than with the modal
    indicator."""
    nx, ny = 128, 8
    params, lo, hi, info = S.train_two_rounds(30, 11, nx=nx, ny=ny, N=3, steps=150, epochs=40, batch=2048)
    assert info["dropped"] == 0
    assert info["loss_round2"][-1] < 0.5 * info["loss_round2"][0]
    desc, kw = S.shock_case(nx, ny, 3)
    g = hg.GpuDGSEM(desc, **kw)
    rng = np.random.default_rng(2024)
    for _ in range(2):
        xs, amp = S.snap_to_face(5.0 + rng.uniform(-0.5, 0.5), nx), rng.uniform(0.1, 0.3)
        stats = {}
        for name, kind in (("modal", hg.SENSOR_MODAL), ("learned", hg.SENSOR_LEARNED)):
            if kind == hg.SENSOR_LEARNED:
                g.set_sensor(kind, mlp=params, lo=lo, hi=hi)
            else:
                g.set_sensor(kind)
            g.set_state(S.shock_state(desc, xs, amp))
            g.time_steps(hg.SCHEME_RK3, 300, 0.0, info["dt"])
            Q = g.state()
            assert np.all(np.isfinite(Q))
            _, out = g.sensor_eval()
            stats[name] = S.shock_metrics(Q, out[:, 3], nx, ny, xs)
            if kind == hg.SENSOR_LEARNED:
                stats["disagreement"] = S.disagreement(out[:, 0], out[:, 3])
        assert stats["learned"]["recall"] >= 0.9
        assert stats["learned"]["recall"] >= stats["modal"]["recall"] + 0.3
        assert stats["learned"]["false_positive_rate"] <= 0.05
        assert stats["learned"]["band_offset"] <= 0.3
        # the shock of the solution stays where it stood at least as well as with the modal indicator
        print(f"shock position error: learned {stats['learned']['shock_position_error']:.3e}, "
              f"modal {stats['modal']['shock_position_error']:.3e}")
        assert stats["learned"]["shock_position_error"] <= stats["modal"]["shock_position_error"] * 1.02 + 1e-6
        assert stats["disagreement"] <= 0.1
