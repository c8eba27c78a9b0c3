"""CPU FP64 restatement of the learned shock sensor (TEST INFRASTRUCTURE: the checker of the GPU
kernels in horses2d_b200/csrc/hg_sensor.cuh and hg_mlp.cu; never called by the product path).

Network: 16 -> 32 -> 32 -> 1, tanh hidden layers, sigmoid output; parameters flattened as
W1[32][16] b1[32] W2[32][32] b2[32] W3[32] b3.  Loss: mean weighted binary cross-entropy on the
logit, w (softplus(z) - t z).  Features of an element: for rho and p, log10 of the fraction of the
modal energy (orthonormal Legendre basis of [0,1]) in modal index k = 0..3 along xi and along eta,
higher indices folded into 3, floored at 1e-10.  No reference counterpart exists.
"""
import numpy as np

N_IN, N_H = 16, 32
SHAPES = [("W1", (N_H, N_IN)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)), ("W3", (N_H,)), ("b3", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def forward(params, X):
    P = unpack(params)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.tanh(X @ P["W1"].T + P["b1"])
    h2 = np.tanh(h1 @ P["W2"].T + P["b2"])
    z = h2 @ P["W3"] + P["b3"][0]
    return z, h1, h2


def predict(params, X):
    z, _, _ = forward(params, X)
    return 1.0 / (1.0 + np.exp(-z))


def loss_grad(params, X, t, w=None):
    """Mean weighted BCE-with-logits and its gradient (flattened like params)."""
    P = unpack(params)
    X = np.asarray(X, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    w = np.ones_like(t) if w is None else np.asarray(w, dtype=np.float64)
    n = len(t)
    z, h1, h2 = forward(params, X)
    loss = np.sum(w * (np.maximum(z, 0) - z * t + np.log1p(np.exp(-np.abs(z))))) / n
    y = 1.0 / (1.0 + np.exp(-z))
    dz = w * (y - t) / n
    gW3 = h2.T @ dz
    gb3 = np.array([dz.sum()])
    a2 = np.outer(dz, P["W3"]) * (1.0 - h2 * h2)
    gW2 = a2.T @ h1
    gb2 = a2.sum(0)
    a1 = (a2 @ P["W2"]) * (1.0 - h1 * h1)
    gW1 = a1.T @ X
    gb1 = a1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, gb3])


def modal_matrix(xi):
    """Inverse of V(i,k) = sqrt(2k+1) L_k(2 xi_i - 1)."""
    P = len(xi)
    V = np.zeros((P, P))
    for k in range(P):
        V[:, k] = np.sqrt(2 * k + 1) * np.polynomial.legendre.legval(2 * np.asarray(xi) - 1, [0] * k + [1])
    return np.linalg.inv(V)


def element_features(Q, xi, gamma=1.4):
    """Features [n_el, 16] and modal indicator s [n_el] from Q [n_el, P*P, 4] (node j*P+i)."""
    P = len(xi)
    Vinv = modal_matrix(xi)
    Q = np.asarray(Q, dtype=np.float64).reshape(-1, P, P, 4)     # [e, j, i, v]
    rho = Q[..., 0]
    p = (gamma - 1.0) * (Q[..., 3] - 0.5 * (Q[..., 1] ** 2 + Q[..., 2] ** 2) / Q[..., 0])
    feats, smax = [], np.full(Q.shape[0], -np.inf)
    for u in (rho, p):
        c = np.einsum("nj,mi,eji->enm", Vinv, Vinv, u)          # c[e, n(eta), m(xi)]
        c2 = c * c
        E = c2.sum((1, 2))
        EN = c2[:, -1, :].sum(1) + c2[:, :-1, -1].sum(1)
        s = np.where((E > 0) & (EN > 0), np.log10(np.maximum(EN, 1e-300) / np.maximum(E, 1e-300)), -np.inf)
        smax = np.maximum(smax, s)
        fold = lambda a: np.concatenate([a[:, :3], a[:, 3:].sum(1, keepdims=True)], 1) if a.shape[1] > 3 else \
            np.concatenate([a, np.zeros((a.shape[0], 4 - a.shape[1]))], 1)
        Ex = fold(c2.sum(1))      # by xi index m
        Ey = fold(c2.sum(2))      # by eta index n
        with np.errstate(divide="ignore", invalid="ignore"):
            fx = np.log10(np.maximum(np.where(E[:, None] > 0, Ex / E[:, None], 0.0), 1e-10))
            fy = np.log10(np.maximum(np.where(E[:, None] > 0, Ey / E[:, None], 0.0), 1e-10))
        feats += [fx, fy]
    return np.concatenate(feats, 1), smax


def ramp(s, s0, kappa):
    return np.where(s < s0 - kappa, 0.0, np.where(s < s0 + kappa, 0.5 * np.sin(0.5 * np.pi * (s - s0) / kappa) + 0.5, 1.0))


def gauss_nodes(P):
    """Legendre-Gauss nodes on [0,1] (numpy's Golub-Welsch nodes; the checker needs no bitwise match)."""
    x, _ = np.polynomial.legendre.leggauss(P)
    return 0.5 * (x + 1.0)


LEARNED_CUT = 0.05


def learned_g(y, cut=LEARNED_CUT):
    """The indicator's G from the network's sigmoid output y: max(0, (y - cut) / (1 - cut))."""
    y = np.asarray(y, dtype=np.float64)
    return np.where(y > cut, (y - cut) / (1.0 - cut), 0.0)


def learned_indicator(params, lo, hi, Q, xi, s0, kappa=1.0):
    """Per-element G of the learned indicator, as the device forms it (hg_sensor.cuh element_sensor):
    learned_g of the network's sigmoid output on the element's 16 features, or the modal-decay G (sine
    ramp of the modal indicator around s0, half width kappa) where a feature, rounded to FP32, lies
    outside the training box [lo, hi] (the out-of-distribution fallback).  FP64 throughout."""
    X, s = element_features(Q, xi)
    g_modal = ramp(s, s0, kappa)
    X32 = X.astype(np.float32)
    ood = np.any((X32 < np.asarray(lo, np.float32)) | (X32 > np.asarray(hi, np.float32)), axis=1)
    return np.where(ood, g_modal, learned_g(predict(params, X))), ood


def step_learned(orc, params, lo, hi, xi, scheme, t, dt, s0, kappa=1.0):
    """One time step of an oracle built with the external indicator (IND_EXTERNAL), with G set from the
    learned indicator of the state at the start of the step (the device holds the indicator of the
    step's first stage for the whole step)."""
    P = len(xi)
    G, _ = learned_indicator(params, lo, hi, orc.state().reshape(-1, P * P, 4), xi, s0, kappa)
    orc.set_av_g(G)
    orc.time_step(scheme, t, dt)
