"""Learned shock sensor: case, training data from the plain solver, GPU training, evaluation.

The sensor sets the element artificial viscosity mu_e = Ceps sqrt(Volume)/(N+1) G of the reference's
artificial dissipation (Approximation/DGArtificialDissipation.f90:277-338).  Three indicators give G
(include/horses_gpu.h, hg_set_sensor): the reference's interface jumps, the modal-decay indicator and
the learned one, an MLP on 16 modal features trained here on the GPU by the library's own kernels
(hg_mlp_train) and evaluated inside the gradient kernel, with the modal indicator as fallback outside
the training feature box and as the judge.

Case (supersonic shock with an entropy wave): [0,10] x [0,1], a stationary Mach-3 normal shock at
x_s with Rankine-Hugoniot states (upstream rho = p = 1 in the solver's units, u = 3 sqrt(gamma)),
density bump rho = 1 + amp sin(5x) upstream at constant pressure and velocity; Euler walls at
y = 0 and 1, supersonic Dirichlet inflow, newDirichlet (static pressure) outflow; Navier-Stokes
build at Re = 0 with interior penalty (SIPG, penalty 10), HLL fluxes and Laplacian artificial
dissipation, as the reference's ShockWave case sets them up.

Ground truth of a snapshot: per row of elements, the shock sits in the first element whose mean
pressure exceeds the mean of the two Rankine-Hugoniot pressures; that element and its two
x-neighbours are troubled (label 1), every other element is smooth (label 0).
"""
import numpy as np

from . import _lib as L
from . import mesh as hmesh
from .solver import GpuDGSEM

GAMMA = 1.4
HARD_WEIGHT = 4.0   # weight of the smooth elements next to the shock band in training (hard negatives)


def rankine_hugoniot(mach, gamma=GAMMA):
    """(rho, u, p) upstream and downstream of a stationary normal shock; upstream rho = p = 1."""
    m2 = mach * mach
    r = (gamma + 1.0) * m2 / ((gamma - 1.0) * m2 + 2.0)
    pr = 1.0 + 2.0 * gamma / (gamma + 1.0) * (m2 - 1.0)
    u1 = mach * np.sqrt(gamma)
    return (1.0, u1, 1.0), (r, u1 / r, pr)


def conservative(rho, u, p, gamma=GAMMA):
    rho, u, p = np.broadcast_arrays(np.asarray(rho, float), np.asarray(u, float), np.asarray(p, float))
    return np.stack([rho, rho * u, 0.0 * rho, p / (gamma - 1.0) + 0.5 * rho * u * u], -1)


def shock_case(nx=512, ny=64, N=3, mach=3.0, node_type=L.NODES_LG, intensity=1.0):
    """(descriptor, GpuDGSEM keyword arguments) of the shock / entropy-wave case."""
    desc = hmesh.box_descriptor(nx, ny, 0.0, 10.0, 0.0, 1.0, N, node_type)
    (r1, u1, p1), (r2, u2, p2) = rankine_hugoniot(mach)
    qin, qout = conservative(r1, u1, p1), conservative(r2, u2, p2)
    kw = dict(mach=mach, reynolds=0.0, navier_stokes=1, viscous=L.IP, ip_method=L.SIPG, sigma0_ip=10.0,
              node_type=node_type, riemann=L.HLL, av_type=L.AV_LAPLACIAN, av_intensity=intensity,
              bcs=[dict(type=L.BC_EULERWALL), dict(type=L.BC_EULERWALL),
                   dict(type=L.BC_DIRICHLET, state=qin), dict(type=L.BC_NEWDIRICHLET, state=qout)])
    return desc, kw


def shock_state(desc, x_shock=5.0, amp=0.2, mach=3.0):
    """Initial state [n_nodes*4] of the case."""
    x = desc["x"].reshape(-1, 2)[:, 0]
    (r1, u1, p1), (r2, u2, p2) = rankine_hugoniot(mach)
    up = x < x_shock
    return conservative(np.where(up, r1 + amp * np.sin(5.0 * x), r2), np.where(up, u1, u2),
                        np.where(up, p1, p2)).ravel()


def snap_to_face(x_shock, nx, x0=0.0, x1=10.0):
    """Shock position moved to the nearest element face (an initial jump inside an element starts the
    run with a discontinuous polynomial, which no indicator damps in time at Mach 3)."""
    h = (x1 - x0) / nx
    return x0 + h * round((x_shock - x0) / h)


def element_pressure(Q, n_el, gamma=GAMMA):
    q = np.asarray(Q).reshape(n_el, -1, 4)
    p = (gamma - 1.0) * (q[..., 3] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2) / q[..., 0])
    return p.mean(1)


def shock_labels(Q, nx, ny, mach=3.0):
    """(labels [n_el] in {0,1}, shock element index per row [ny]) of a state (box element order)."""
    (_, _, p1), (_, _, p2) = rankine_hugoniot(mach)
    pm = element_pressure(Q, nx * ny).reshape(ny, nx)
    lab = np.zeros((ny, nx))
    col = np.argmax(pm > 0.5 * (p1 + p2), axis=1)
    for j in range(ny):
        lab[j, max(col[j] - 1, 0):min(col[j] + 2, nx)] = 1.0
    return lab.ravel(), col


def generate_snapshots(n_snap, seed, nx=512, ny=64, N=3, steps=200, cfl=0.1, precision=L.PREC_FP64,
                       neg_ratio=8, learned=None, hard_weight=None):
    """Plain-solver snapshots (modal-decay sensor) of seeded shock positions x_s = 5 + U(-0.5, 0.5)
    (moved to the nearest element face) and bump amplitudes U(0.1, 0.3).  Returns a dict with the
    sampled training set (all troubled elements, the smooth elements two to four elements from the
    band on either side, and neg_ratio times as many other smooth ones per snapshot, each also with
    the element's axes swapped; class-balanced
    weights, the near-band smooth elements weighted hard_weight times more); snapshots whose state is not
    finite are left out and counted.
    learned = (params, lo, hi) runs the solver with the learned indicator instead (the second round
    of training sees the states the learned sensor itself produces)."""
    hard_weight = HARD_WEIGHT if hard_weight is None else hard_weight
    rng = np.random.default_rng(seed)
    desc, kw = shock_case(nx, ny, N)
    g = GpuDGSEM(desc, precision=precision, **kw)
    if learned is None:
        g.set_sensor(L.SENSOR_MODAL)
    else:
        g.set_sensor(L.SENSOR_LEARNED, mlp=learned[0], lo=learned[1], hi=learned[2])
    g.set_state(shock_state(desc))
    dt = g.estimate_time_step(cfl, 1.0)
    Xs, ts, hs, meta = [], [], [], []
    dropped = 0
    for _ in range(n_snap):
        xs, amp = snap_to_face(5.0 + rng.uniform(-0.5, 0.5), nx), rng.uniform(0.1, 0.3)
        g.set_state(shock_state(desc, xs, amp))
        g.time_steps(L.SCHEME_RK3, steps, 0.0, dt)
        Q = g.state()
        if not np.all(np.isfinite(Q)):
            dropped += 1
            continue
        feats, _ = g.sensor_eval()
        lab, col = shock_labels(Q, nx, ny)
        pos = np.flatnonzero(lab > 0.5)
        # hard negatives: the smooth cells two to four elements from the labelled band on either side
        # (the post-shock oscillation makes the downstream ones look troubled), always in the set
        off = np.array([-4, -3, -2, 2, 3, 4])
        near = (np.arange(ny)[:, None] * nx + np.clip(col[:, None] + off[None, :], 0, nx - 1)).ravel()
        near = np.unique(near[lab[near] < 0.5])
        neg = np.setdiff1d(np.flatnonzero(lab < 0.5), near)
        neg = rng.choice(neg, size=min(len(neg), neg_ratio * len(pos)), replace=False)
        idx = np.concatenate([pos, near, neg])
        hard = np.concatenate([np.zeros(len(pos)), np.ones(len(near)), np.zeros(len(neg))])
        # every sample also with the element's axes swapped (the shock along eta), so that the network
        # and its feature box see both directions of a flow that is 1D here
        Xs += [feats[idx], transpose_features(feats[idx])]
        ts += [lab[idx], lab[idx]]
        hs += [hard, hard]
        meta.append((xs, amp))
    X = np.concatenate(Xs).astype(np.float32)
    t = np.concatenate(ts).astype(np.float32)
    hard = np.concatenate(hs)
    w = sample_weights(t, hard, hard_weight)
    g.close()
    return dict(X=X, t=t, w=w, hard=hard, meta=meta, dt=dt, steps=steps, dropped=dropped)


def transpose_features(X):
    """Features of the same elements with xi and eta swapped (per variable: the four xi-index
    fractions trade places with the four eta-index ones)."""
    X = np.asarray(X)
    return X[:, [4, 5, 6, 7, 0, 1, 2, 3, 12, 13, 14, 15, 8, 9, 10, 11]]


def sample_weights(t, hard, hard_weight=HARD_WEIGHT):
    """Class-balanced weights (each class sums to half), the near-band smooth samples hard_weight times
    heavier."""
    w = np.where(t > 0.5, 0.5 / max(t.mean(), 1e-12), 0.5 / max(1.0 - t.mean(), 1e-12))
    return (w * np.where(hard > 0.5, hard_weight, 1.0)).astype(np.float32)


def train_two_rounds(n_snap, seed, nx=512, ny=64, N=3, steps=200, epochs=40, batch=4096, lr=2e-3):
    """Round 1: snapshots of the plain solver (modal indicator), train.  Round 2: snapshots of the
    solver driven by the round-1 network, train again on the union.  Returns (params, lo, hi, info)."""
    d1 = generate_snapshots(n_snap, seed, nx, ny, N, steps)
    p1, h1 = train(d1["X"], d1["t"], d1["w"], epochs, batch, lr, seed)
    lo, hi = feature_box(d1["X"])
    d2 = generate_snapshots(n_snap, seed + 1, nx, ny, N, steps, learned=(p1, lo, hi))
    X = np.concatenate([d1["X"], d2["X"]])
    t = np.concatenate([d1["t"], d2["t"]])
    w = sample_weights(t, np.concatenate([d1["hard"], d2["hard"]]))
    p2, h2 = train(X, t, w, epochs, batch, lr, seed + 1)
    lo, hi = feature_box(X)
    return p2, lo, hi, dict(samples=len(t), dropped=d1["dropped"] + d2["dropped"], loss_round1=h1.tolist(),
                            loss_round2=h2.tolist(), dt=d1["dt"])


def init_params(seed):
    """Xavier-uniform weights, zero biases (W1 b1 W2 b2 W3 b3)."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((16, 32), (32, 32), (32, 1)):
        a = np.sqrt(6.0 / (fan_in + fan_out))
        parts += [rng.uniform(-a, a, fan_in * fan_out), np.zeros(fan_out)]
    return np.concatenate(parts).astype(np.float32)


def train(X, t, w=None, epochs=20, batch=4096, lr=2e-3, seed=0):
    """GPU training (hg_mlp_train).  Returns (params float32[1633], per-epoch loss)."""
    lib = L.load()
    p = init_params(seed)
    X = np.ascontiguousarray(X, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    wp = None if w is None else np.ascontiguousarray(w, np.float32)
    hist = np.zeros(epochs)
    rc = lib.hg_mlp_train(p.ctypes.data_as(L.F32P), X.ctypes.data_as(L.F32P), t.ctypes.data_as(L.F32P),
                          None if wp is None else wp.ctypes.data_as(L.F32P), len(t), epochs, batch, lr, seed,
                          hist.ctypes.data_as(L.F64P))
    if rc != 0:
        raise RuntimeError(f"hg_mlp_train failed ({rc})")
    return p, hist


def feature_box(X, margin=0.1, pad=0.5):
    """Per-feature [lo, hi] of the training set widened by margin * span + pad (features are log10)."""
    lo, hi = X.min(0), X.max(0)
    d = margin * (hi - lo) + pad
    return (lo - d).astype(np.float32), (hi + d).astype(np.float32)


def mlp_forward(params, X):
    lib = L.load()
    X = np.ascontiguousarray(X, np.float32)
    y = np.zeros(len(X), np.float32)
    p = np.ascontiguousarray(params, np.float32)
    if lib.hg_mlp_forward(p.ctypes.data_as(L.F32P), X.ctypes.data_as(L.F32P), len(X), y.ctypes.data_as(L.F32P)):
        raise RuntimeError("hg_mlp_forward failed")
    return y


def mlp_grad(params, X, t, w=None):
    lib = L.load()
    X = np.ascontiguousarray(X, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    p = np.ascontiguousarray(params, np.float32)
    wp = None if w is None else np.ascontiguousarray(w, np.float32)
    g = np.zeros(L.MLP_PARAMS, np.float32)
    loss = np.zeros(1)
    rc = lib.hg_mlp_grad(p.ctypes.data_as(L.F32P), X.ctypes.data_as(L.F32P), t.ctypes.data_as(L.F32P),
                         None if wp is None else wp.ctypes.data_as(L.F32P), len(t), loss.ctypes.data_as(L.F64P),
                         g.ctypes.data_as(L.F32P))
    if rc != 0:
        raise RuntimeError(f"hg_mlp_grad failed ({rc})")
    return float(loss[0]), g


TROUBLED = 0.05   # an element is troubled when its indicator G reaches 5 % of the maximum viscosity


def shock_crossing(Q, nx, ny, mach=3.0, x0=0.0, x1=10.0):
    """Shock position of a state per row of elements: where the pressure profile along x (nodal
    pressures averaged over each element's eta nodes, at the Legendre-Gauss nodes) first reaches the
    mean of the Rankine-Hugoniot pressures, linearly interpolated between nodes."""
    (_, _, p1), (_, _, p2) = rankine_hugoniot(mach)
    q = np.asarray(Q, dtype=np.float64)
    P = int(round(np.sqrt(q.size // (4 * nx * ny))))
    q = q.reshape(ny, nx, P, P, 4)
    p = (GAMMA - 1.0) * (q[..., 3] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2) / q[..., 0])
    prof = p.mean(2).reshape(ny, nx * P)
    xi = 0.5 * (np.polynomial.legendre.leggauss(P)[0] + 1.0)
    xs = (x0 + (x1 - x0) / nx * (np.arange(nx)[:, None] + xi[None, :])).ravel()
    mid = 0.5 * (p1 + p2)
    k = np.maximum(np.argmax(prof > mid, axis=1), 1)
    r = np.arange(ny)
    pa, pb = prof[r, k - 1], prof[r, k]
    return xs[k - 1] + (mid - pa) / (pb - pa) * (xs[k] - xs[k - 1])


def shock_metrics(Q, G, nx, ny, x_shock, mach=3.0, x0=0.0, x1=10.0, thr=TROUBLED):
    """Troubled-cell statistics of one indicator G on a state against the pressure-jump ground truth:
    recall, false-positive rate more than 3 elements from the shock, the shock position error of the
    solution (mean over rows of |shock_crossing - x_shock|: the case is a standing shock started at
    x_shock, so the dissipation that the indicator adds is what moves it), the offset of the troubled
    band (G-weighted x-centroid of the troubled cells against the centre of the labelled band, per
    row) and the pressure overshoot away from the shock (max |p - p_RH| / p_RH more than 3 elements
    off the shock)."""
    (_, _, p1), (_, _, p2) = rankine_hugoniot(mach)
    lab, col = shock_labels(Q, nx, ny, mach)
    h = (x1 - x0) / nx
    xc = x0 + h * (np.arange(nx) + 0.5)
    Gm = np.asarray(G).reshape(ny, nx)
    fl = Gm >= thr
    labm = lab.reshape(ny, nx) > 0.5
    dist = np.arange(nx)[None, :] - col[:, None]
    far = np.abs(dist) > 3
    offs = []
    for j in range(ny):
        wj = np.where(fl[j], Gm[j], 0.0)
        offs.append(abs((wj * xc).sum() / wj.sum() - xc[col[j]]) if wj.sum() > 0 else x1 - x0)
    pm = element_pressure(Q, nx * ny).reshape(ny, nx)
    pref = np.where(dist < 0, p1, p2)
    over = np.abs(pm - pref) / pref
    return dict(recall=float((fl & labm).sum() / max(labm.sum(), 1)),
                false_positive_rate=float((fl & far).sum() / max(far.sum(), 1)),
                troubled=int(fl.sum()),
                shock_position_error=float(np.mean(np.abs(shock_crossing(Q, nx, ny, mach, x0, x1) - x_shock))),
                band_offset=float(np.mean(offs)), pressure_overshoot=float(over[far].max()))


def disagreement(g_a, g_b, thr=TROUBLED):
    """Fraction of elements that one indicator calls troubled and the other does not."""
    return float(np.mean((np.asarray(g_a) >= thr) != (np.asarray(g_b) >= thr)))
