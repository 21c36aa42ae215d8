"""FP64 CPU restatement of the learned scheduler's MLP and training loss.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA training kernels in
medusa_b200/csrc/learn.cu (k_mlp_grad) and the inference in
medusa_b200/csrc/sched.cuh (mlp_pick_warp).  No reference counterpart: the
reference has one fixed schedule.

Layout of the parameter vector (row-major): w1[32][6], b1[32], w2[32][32],
b2[32], w3[8][32], b3[8].  Loss per sample: cross-entropy between the
softmax of the outputs and the target q_s ~ exp(-(t_s - t_min)/(0.25 t_min))
over the measured schedules (t_s > 0); the batch loss and gradient are
means weighted by each sample's best time, w_i = t_min,i / sum_j t_min,j.
Features (sched.cuh make_features): log2(1+count)/32 for frontier vertices,
frontier out-edges, unvisited vertices and unvisited out-edges; degree skew
log2(max/mean out-degree)/16 (capped at 1); frontier format 0/1.
"""
import numpy as np

F, H, O = 6, 32, 8
TAU = 0.25
SIZES = [("w1", (H, F)), ("b1", (H,)), ("w2", (H, H)), ("b2", (H,)), ("w3", (O, H)), ("b3", (O,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(P):
    out, i = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(P[i:i + n], np.float64).reshape(shape)
        i += n
    return out


def pack(d):
    return np.concatenate([d[name].reshape(-1) for name, _ in SIZES])


def targets(T):
    T = np.asarray(T, np.float64)
    valid = T > 0
    tmin = np.where(valid, T, np.inf).min(axis=1, keepdims=True)
    q = np.where(valid, np.exp(-(T - tmin) / (TAU * tmin)), 0.0)
    z = q.sum(axis=1, keepdims=True)
    return np.where(z > 0, q / np.where(z > 0, z, 1), 0.0)


def features(n, m, nu, mu, skew, mode):
    f = np.log2(1.0 + np.array([n, m, max(nu, 0), max(mu, 0)], np.float64)) / 32
    return np.concatenate([f, [min(skew, 16.0) / 16.0, float(mode)]])


def weights(T):
    T = np.asarray(T, np.float64)
    tmin = np.where(T > 0, T, np.inf).min(axis=1)
    w = np.where(np.isfinite(tmin), tmin, 0.0)
    s = w.sum()
    return w / s if s > 0 else w


def forward(P, X):
    w = unpack(P)
    X = np.asarray(X, np.float64)
    z1 = X @ w["w1"].T + w["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w["w2"].T + w["b2"]
    h2 = np.maximum(z2, 0)
    o = h2 @ w["w3"].T + w["b3"]
    return z1, h1, z2, h2, o


def loss_and_grad(P, X, T):
    w = unpack(P)
    X = np.asarray(X, np.float64)
    z1, h1, z2, h2, o = forward(P, X)
    o = o - o.max(axis=1, keepdims=True)
    p = np.exp(o)
    p /= p.sum(axis=1, keepdims=True)
    q = targets(T)
    sw = weights(T)[:, None]
    loss = -(sw * q * np.log(np.maximum(p, 1e-30))).sum()
    do = (p - q) * sw
    g = {"w3": do.T @ h2, "b3": do.sum(0)}
    dz2 = (do @ w["w3"]) * (z2 > 0)
    g["w2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ w["w2"]) * (z1 > 0)
    g["w1"] = dz1.T @ X
    g["b1"] = dz1.sum(0)
    return loss, pack(g)


OVERRIDE_MARGIN = 1.0
BOUNDS_SLACK = 1.0 / 32


def pick(P, X, fallback=None, bounds=None):
    """argmax of the outputs; with fallback, keep fallback[i] unless the
    row's features lie within bounds = (lo[6], hi[6]) +- BOUNDS_SLACK (None:
    unbounded) and the best output beats the fallback's by more than
    OVERRIDE_MARGIN."""
    X = np.asarray(X, np.float64)
    o = forward(P, X)[4]
    best = o.argmax(axis=1)
    if fallback is None:
        return best
    fb = np.asarray(fallback)
    idx = np.arange(len(o))
    ok = o[idx, best] - o[idx, fb] > OVERRIDE_MARGIN
    if bounds is not None:
        lo, hi = (np.asarray(b, np.float64) for b in bounds)
        ok &= ((X >= lo - BOUNDS_SLACK) & (X <= hi + BOUNDS_SLACK)).all(axis=1)
    return np.where(ok, best, fb)
