"""CPU oracle of the warm-start MLP (test infrastructure only).

Restates, in numpy, the network the tensor-core kernels compute: 8 inputs
(padded to 16) -> 128 -> 128 -> 128 (SiLU) -> 5 outputs (padded to 16), no
bias other than the constant input; loss mean((y - t)^2) over the 5 outputs;
Adam with beta 0.9 / 0.999, eps 1e-8.  The weight vector has 36864 entries in
the order W1[128][16], W2[128][128], W3[128][128], W4[16][128].

Two modes:
  ``exact``  float64 throughout -- pinned against finite differences;
  ``kernel`` rounds to bf16 where the kernels do (inputs, weights, each
             activation, dY and each dZ before it enters a GEMM) and
             accumulates in float64, so that it differs from the kernels only
             by accumulation order and the hardware tanh used for the sigmoid.

The network has no counterpart in the reference (it is new in this
implementation); the solver fields it is trained on follow the reference's
PhysicsEuler (src/models/euler.cu).
"""
from __future__ import annotations

import numpy as np

N_IN, N_FEAT, N_HID, N_OUT_PAD, N_OUT = 16, 8, 128, 16, 5
OFF_W1 = 0
OFF_W2 = OFF_W1 + N_HID * N_IN
OFF_W3 = OFF_W2 + N_HID * N_HID
OFF_W4 = OFF_W3 + N_HID * N_HID
N_PARAMS = OFF_W4 + N_OUT_PAD * N_HID


def bf16(x):
    """Round float32 values to bf16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(np.shape(x))


def split(w):
    w = np.asarray(w)
    return (w[OFF_W1:OFF_W2].reshape(N_HID, N_IN), w[OFF_W2:OFF_W3].reshape(N_HID, N_HID),
            w[OFF_W3:OFF_W4].reshape(N_HID, N_HID), w[OFF_W4:].reshape(N_OUT_PAD, N_HID))


def join(w1, w2, w3, w4):
    return np.concatenate([w1.ravel(), w2.ravel(), w3.ravel(), w4.ravel()])


def padding_mask():
    """True where a weight multiplies an input padding column or feeds a padding output."""
    m = np.zeros(N_PARAMS, bool)
    m1, _, _, m4 = split(m)
    m1[:, N_FEAT:] = True
    m4[N_OUT:, :] = True
    return m


def sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * sigmoid(z)


def dsilu(z):
    s = sigmoid(z)
    return s * (1.0 + z * (1.0 - s))


def _round(x, mode):
    return bf16(x).astype(np.float64) if mode == "kernel" else np.asarray(x, np.float64)


def forward(w, x, mode="exact"):
    """x[n][8] -> (y[n][5], cache)."""
    w1, w2, w3, w4 = (_round(m, mode) for m in split(w))
    n = x.shape[0]
    xp = np.zeros((n, N_IN))
    xp[:, :N_FEAT] = x
    xp = _round(xp, mode)
    z1 = xp @ w1.T
    a1 = _round(silu(z1), mode)
    z2 = a1 @ w2.T
    a2 = _round(silu(z2), mode)
    z3 = a2 @ w3.T
    a3 = _round(silu(z3), mode)
    y = a3 @ w4.T
    return y[:, :N_OUT], (xp, z1, a1, z2, a2, z3, a3, y, (w1, w2, w3, w4))


def loss_and_grad(w, x, t, mode="exact"):
    """Loss mean((y - t)^2) and its gradient w.r.t. the 36864 weights."""
    y, (xp, z1, a1, z2, a2, z3, a3, yf, (w1, w2, w3, w4)) = forward(w, x, mode)
    n = x.shape[0]
    e = y - t
    loss = float(np.mean(e * e))
    dy = np.zeros((n, N_OUT_PAD))
    dy[:, :N_OUT] = (2.0 / (n * N_OUT)) * e
    dy = _round(dy, mode)
    g4 = dy.T @ a3
    da3 = dy @ w4
    dz3 = _round(da3 * dsilu(z3), mode)
    g3 = dz3.T @ a2
    da2 = dz3 @ w3
    dz2 = _round(da2 * dsilu(z2), mode)
    g2 = dz2.T @ a1
    da1 = dz2 @ w2
    dz1 = _round(da1 * dsilu(z1), mode)
    g1 = dz1.T @ xp
    return loss, join(g1, g2, g3, g4)


def adam_step(w, m, v, g, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (step counts from 1); padding weights stay untouched."""
    keep = padding_mask()
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    nw = w - lr * mh / (np.sqrt(vh) + eps)
    nw[keep] = w[keep]
    return nw, m, v


def init_like_kernel(seed_rng: np.random.Generator):
    """A random weight vector with the kernels' padding zeros (not the kernels' own init)."""
    w = np.zeros(N_PARAMS)
    w1, w2, w3, w4 = split(w)
    w1[:, :N_FEAT] = seed_rng.uniform(-1, 1, (N_HID, N_FEAT)) / np.sqrt(N_FEAT)
    w2[:] = seed_rng.uniform(-1, 1, (N_HID, N_HID)) / np.sqrt(N_HID)
    w3[:] = seed_rng.uniform(-1, 1, (N_HID, N_HID)) / np.sqrt(N_HID)
    w4[:N_OUT] = seed_rng.uniform(-1, 1, (N_OUT, N_HID)) / np.sqrt(N_HID)
    return w


# ---- input features ----
def squash(u):
    return u / np.sqrt(1.0 + u * u)


def point_triangle_distance(p, a, b, c):
    """Distance from points p[n][3] to triangle (a, b, c): minimum over the
    triangle's interior (barycentric projection) and its three edges."""
    p = np.asarray(p, np.float64)
    ab, ac = b - a, c - a
    nrm = np.cross(ab, ac)
    nn = nrm @ nrm
    best = np.full(len(p), np.inf)
    if nn > 0:
        ap = p - a
        # barycentric coordinates of the projection
        d00, d01, d11 = ab @ ab, ab @ ac, ac @ ac
        d20, d21 = ap @ ab, ap @ ac
        den = d00 * d11 - d01 * d01
        v = (d11 * d20 - d01 * d21) / den
        w = (d00 * d21 - d01 * d20) / den
        inside = (v >= 0) & (w >= 0) & (v + w <= 1)
        h = np.abs(ap @ nrm) / np.sqrt(nn)
        best = np.where(inside, h, best)
    for s0, s1 in ((a, b), (b, c), (c, a)):
        d = s1 - s0
        tt = np.clip(((p - s0) @ d) / max(d @ d, 1e-300), 0.0, 1.0)
        q = s0 + tt[:, None] * d
        best = np.minimum(best, np.linalg.norm(p - q, axis=1))
    return best


def geometry_features(centroids, wall_faces, centre, length):
    """(x', y', z', d') per cell: squash((x - centre) / length) and
    squash(distance to the nearest wall triangle / length); wall_faces is a
    list of node-coordinate arrays, fan-triangulated."""
    d = np.full(len(centroids), np.inf)
    for f in wall_faces:
        for k in range(1, len(f) - 1):
            d = np.minimum(d, point_triangle_distance(centroids, f[0], f[k], f[k + 1]))
    u = (np.asarray(centroids, np.float64) - centre) / length
    return np.column_stack([squash(u), squash(d / length)])
