"""CPU oracle for the learned troubled-cell indicator (numpy, float64).

TEST INFRASTRUCTURE ONLY: tests/ use it to check the library's feature, MLP forward, gradient and Adam
kernels. The indicator has no counterpart in the reference; its label is the reference limiter's own
decision (CS_slope_limiter_serial, source/problem/SWE/problem_slope_limiter/swe_CS_slope_limiter.hpp:89-189:
a cell is troubled when the Cockburn-Shu pass changes its state), and its inputs are the quantities
that limiter reads: the linear modal coefficients of ze, qx, qy and the three neighbour cell means.

Features (18 per element, p = 1). The limiter compares, per median direction, characteristic slopes
w = R^-1 q of the cell with R^-1-weighted neighbour differences, where R^-1 mixes ze with q / c
(c = sqrt(g H)) and the Froude number u / c, and leaves a slope alone when it is below M r^2 (TVB).
So the fields are first put in common units: ze as is, qx and qy divided by the cell's c; then
a = own mean (mode 0), b, c = modes 1, 2, d_f = (neighbour mean across face f) - a (0 at a boundary),
and one scale s = max over the three fields of |b|, |c|, |d_f| (1 where that is 0):
  [0]  s / (s + M r2)            r2 = mean squared centroid-to-edge-midpoint distance (TVB ratio)
  [1]  clamp(u / c, -8, 8)       u = qx_mean / H, H = max(ze_mean + b_c, 1e-3), b_c = mean vertex depth
  [2]  clamp(v / c, -8, 8)
  [3 + 5 v + 0, 1]  b / s, c / s of field v
  [3 + 5 v + 2 + f] d_f / s
A cell takes part (ok) when it and its three neighbours are wet and each boundary face is land or
function, the same condition under which the limiter looks at it.

Feature set 1 ("raw", the learned-indicator workload's literal input list): [3 v + k] the modal
coefficient k = 0, 1, 2 of field v (ze, qx, qy), then [9 + 3 f + v] the cell mean of field v in the
neighbour across face f (the cell's own mean at a boundary face).

Parameter vector (FP32 master copy, 5441 values): W1[64][18], b1[64], W2[64][64], b2[64], w3[64], b3.
"""
import numpy as np

N_IN, N_H = 18, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_H * N_IN
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_H
N_PARAM = OFF_B3 + 1


def unpack(P):
    P = np.asarray(P, np.float64)
    return (P[OFF_W1:OFF_B1].reshape(N_H, N_IN), P[OFF_B1:OFF_W2], P[OFF_W2:OFF_B2].reshape(N_H, N_H),
            P[OFF_B2:OFF_W3], P[OFF_W3:OFF_B3], P[OFF_B3])


def features(q, wet, nbr, btype, node_xyz, elem_nodes, g, M, fset=0):
    """q [ne][3][nd] (ascending element ID), wet [ne], nbr [ne][3] (-1 at boundaries), btype [ne][3],
    node_xyz [nn][3], elem_nodes [ne][3], gravity g, TVB constant M, feature set -> (features [ne][18]
    float32, ok [ne] bool). Operation order matches the device code exactly (no fused multiply-adds)."""
    q = np.asarray(q, np.float64)
    ne = q.shape[0]
    a = q[:, :, 0].copy()
    b = q[:, :, 1].copy()
    c = q[:, :, 2].copy()
    has = nbr >= 0
    m = np.where(has[:, :, None], q[np.where(has, nbr, 0), :, 0], a[:, None, :])  # [ne][face][var]
    w = np.asarray(wet) != 0
    nbr_wet = np.where(has, w[np.where(has, nbr, 0)], btype <= 3)  # land, tide, flow, function objects
    ok = w & nbr_wet.all(axis=1)
    if fset == 1:
        F = np.empty((ne, 18), np.float64)
        F[:, 0:9] = q[:, :, 0:3].reshape(ne, 9)
        F[:, 9:18] = m.reshape(ne, 9)
        return F.astype(np.float32), ok
    d = m - a[:, None, :]
    X = node_xyz[elem_nodes]  # [ne][3][3]
    zb = X[:, 0, 2] * (1.0 / 3.0) + X[:, 1, 2] * (1.0 / 3.0) + X[:, 2, 2] * (1.0 / 3.0)
    H = np.maximum(a[:, 0] + zb, 1e-3)
    ic = 1.0 / np.sqrt(g * H)
    for v in (1, 2):
        b[:, v] = b[:, v] * ic
        c[:, v] = c[:, v] * ic
        d[:, :, v] = d[:, :, v] * ic[:, None]
    s = np.maximum(np.maximum(np.abs(b), np.abs(c)).max(axis=1), np.abs(d).max(axis=(1, 2)))
    s = np.where(s == 0.0, 1.0, s)
    cx = (X[:, 0, 0] + X[:, 1, 0] + X[:, 2, 0]) / 3.0
    cy = (X[:, 0, 1] + X[:, 1, 1] + X[:, 2, 1]) / 3.0
    r2 = np.zeros(ne)
    for k in range(3):
        mx = (X[:, (k + 1) % 3, 0] + X[:, (k + 2) % 3, 0]) / 2.0 - cx
        my = (X[:, (k + 1) % 3, 1] + X[:, (k + 2) % 3, 1]) / 2.0 - cy
        r2 = r2 + (mx * mx + my * my)
    r2 = r2 / 3.0
    inv = 1.0 / s
    F = np.empty((ne, 18), np.float64)
    F[:, 0] = s / (s + M * r2)
    F[:, 1] = np.clip((a[:, 1] / H) * ic, -8.0, 8.0)
    F[:, 2] = np.clip((a[:, 2] / H) * ic, -8.0, 8.0)
    for v in range(3):
        F[:, 3 + 5 * v] = b[:, v] * inv
        F[:, 4 + 5 * v] = c[:, v] * inv
        for f in range(3):
            F[:, 5 + 5 * v + f] = d[:, f, v] * inv
    return F.astype(np.float32), ok


def forward(P, X):
    W1, b1, W2, b2, w3, b3 = unpack(P)
    X = np.asarray(X, np.float64)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    z3 = h2 @ w3 + b3
    return 1.0 / (1.0 + np.exp(-z3)), (z1, h1, z2, h2, z3)


def loss_and_grad(P, X, y, pos_weight):
    """Mean weighted binary cross-entropy -[w y log p + (1 - y) log(1 - p)] and its gradient."""
    W1, b1, W2, b2, w3, b3 = unpack(P)
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)
    n = X.shape[0]
    p, (z1, h1, z2, h2, z3) = forward(P, X)
    wy = pos_weight * y
    # log p = -softplus(-z), log(1-p) = -softplus(z)
    sp_neg = np.logaddexp(0.0, -z3)
    sp_pos = np.logaddexp(0.0, z3)
    loss = np.mean(wy * sp_neg + (1.0 - y) * sp_pos)
    d3 = (p * (1.0 - y) - wy * (1.0 - p)) / n
    g = np.zeros(N_PARAM)
    g[OFF_W3:OFF_B3] = h2.T @ d3
    g[OFF_B3] = d3.sum()
    d2 = np.outer(d3, w3) * (z2 > 0)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(axis=0)
    d1 = (d2 @ W2) * (z1 > 0)
    g[OFF_W1:OFF_B1] = (d1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(axis=0)
    return loss, g


def adam(P, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba 2015, bias-corrected), float64."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return P - lr * mh / (np.sqrt(vh) + eps), m, v


def bf16_round(x):
    """Round float32 values to bfloat16 (round to nearest, ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward_bf16(P, X):
    """The tensor-core inference path: x, W1, W2 and the first hidden layer rounded to bfloat16,
    products accumulated in float64 here (float32 on the device), biases and the output layer exact."""
    W1, b1, W2, b2, w3, b3 = unpack(P)
    W1b = bf16_round(W1).astype(np.float64)
    W2b = bf16_round(W2).astype(np.float64)
    Xb = bf16_round(np.asarray(X, np.float32)).astype(np.float64)
    h1 = np.maximum(Xb @ W1b.T + b1.astype(np.float32), 0.0)
    h1b = bf16_round(h1.astype(np.float32)).astype(np.float64)
    h2 = np.maximum(h1b @ W2b.T + b2.astype(np.float32), 0.0)
    z3 = h2 @ w3 + b3
    return 1.0 / (1.0 + np.exp(-z3))


def init_params(seed):
    """He-uniform weights, zero biases (the training start point)."""
    rng = np.random.default_rng(seed)
    P = np.zeros(N_PARAM, np.float32)
    P[OFF_W1:OFF_B1] = rng.uniform(-1, 1, N_H * N_IN) * np.sqrt(6.0 / N_IN)
    P[OFF_W2:OFF_B2] = rng.uniform(-1, 1, N_H * N_H) * np.sqrt(6.0 / N_H)
    P[OFF_W3:OFF_B3] = rng.uniform(-1, 1, N_H) * np.sqrt(6.0 / N_H)
    return P
