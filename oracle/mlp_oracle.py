"""CPU FP64 oracle of the learned Riemann guess (TEST INFRASTRUCTURE ONLY).

The network has no counterpart in the reference; this file is the CPU
checker of the project's tensor-core kernels: features, forward pass, loss and
the full backward pass in float64 numpy.  With bf16=True it rounds weights,
inputs, hidden activations and back-propagated pre-activation gradients to
bfloat16 at the points where the GPU kernels do, so the remaining difference
is FP32 accumulation order only.
"""
from __future__ import annotations

import numpy as np

H, IN = 64, 5
NPARAM = H * IN + H + 2 * (H * H + H) + H + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W0 = p[o:o + H * IN].reshape(H, IN); o += H * IN
    b0 = p[o:o + H]; o += H
    W1 = p[o:o + H * H].reshape(H, H); o += H * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W0, b0, W1, b1, W2, b2, w3, b3


def pack(W0, b0, W1, b1, W2, b2, w3, b3):
    return np.concatenate([W0.ravel(), b0, W1.ravel(), b1, W2.ravel(), b2, w3, [b3]])


def bf16(x):
    """Round float64 -> float32 -> bfloat16 (nearest even), back to float64."""
    f = np.asarray(x, dtype=np.float32).copy()
    u = f.view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    u = ((u + r) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def features(states):
    """Scaled inputs of rows (u_L, rho_L, p_L, u_R, rho_R, p_R, gamma)."""
    s = np.asarray(states, dtype=np.float64).reshape(-1, 7)
    uL, rL, pL, uR, rR, pR, g = s.T
    cl = np.sqrt(g * pL / rL)
    cr = np.sqrt(g * pR / rR)
    x = np.stack([np.log(rR / rL) * (1.0 / 7.0), np.log(pR / pL) * (1.0 / 9.0), (uR - uL) / cl * 0.2,
                  np.minimum(cr / cl, 64.0) * 0.125, (g - 1.5) * 4.0], axis=1)
    return x.astype(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x, emulate_bf16=False):
    W0, b0, W1, b1, W2, b2, w3, b3 = unpack(p)
    q = bf16 if emulate_bf16 else (lambda a: a)
    a0 = q(x)
    z1 = a0 @ q(W0).T + b0
    a1 = silu(z1)
    z2 = q(a1) @ q(W1).T + b1
    a2 = silu(z2)
    z3 = q(a2) @ q(W2).T + b2
    a3 = silu(z3)
    y = a3 @ w3 + b3
    return y, (a0, z1, a1, z2, a2, z3, a3)


def loss_and_grad(p, x, target, emulate_bf16=False):
    """Mean squared error and its gradient w.r.t. all parameters."""
    W0, b0, W1, b1, W2, b2, w3, b3 = unpack(p)
    q = bf16 if emulate_bf16 else (lambda a: a)
    y, (a0, z1, a1, z2, a2, z3, a3) = forward(p, x, emulate_bf16)
    n = len(y)
    e = y - target
    loss = float(np.mean(e * e))
    dy = 2.0 * e / n
    gw3 = a3.T @ dy
    gb3 = dy.sum()
    dz3 = np.outer(dy, w3) * dsilu(z3)
    gW2 = q(dz3).T @ q(a2)
    gb2 = dz3.sum(0)
    dz2 = (q(dz3) @ q(W2)) * dsilu(z2)
    gW1 = q(dz2).T @ q(a1)
    gb1 = dz2.sum(0)
    dz1 = (q(dz2) @ q(W1)) * dsilu(z1)
    gW0 = q(dz1).T @ a0
    gb0 = dz1.sum(0)
    return loss, pack(gW0, gb0, gW1, gb1, gW2, gb2, gw3, gb3)


def random_states(n, seed=12345):
    """Random Riemann problems: log-uniform p ratio 1e-4..1e4, log-uniform rho
    ratio 1e-3..1e3, velocity jump uniform in +-5 c_L, gamma in {1.4, 5/3}
    (Philox stream of the given seed)."""
    rng = np.random.Generator(np.random.Philox(seed))
    rL = np.ones(n)
    pL = np.ones(n)
    g = np.where(rng.random(n) < 0.5, 1.4, 5.0 / 3.0)
    rR = 10.0 ** rng.uniform(-3, 3, n)
    pR = 10.0 ** rng.uniform(-4, 4, n)
    cl = np.sqrt(g * pL / rL)
    du = rng.uniform(-5, 5, n) * cl
    uL = np.zeros(n)
    uR = du
    return np.stack([uL, rL, pL, uR, rR, pR, g], axis=1)
