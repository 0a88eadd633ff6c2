"""CPU restatement of the learned warm start (test infrastructure only).

ORACLE: only tests/, the smoke check and bench.py's baseline legs use this
module, as the checker of the device kernels; the product never imports it.

The reference has no learned part (it always starts from the Maxwellian at
rest, Initialization/InitialConditions.cpp:18-80), so there is nothing of the
reference to pin here except the 2-D Chu moment sums this module shares with
the step (MomentCalculations/Moments.cpp:66-97) and the Maxwellians
(MLSTransport/MLSBasis.hpp:87-104, g2 = R T g1 / 2).  What it restates:

* the network: 64 features -> 4 tanh layers of width 128 -> 16 outputs, BF16
  weights and activations (round to nearest even), FP32 sums, the same
  rounding points as the tensor-core kernels;
* its backward pass and Adam, in FP32 as the kernels do them, and an FP64
  version without rounding for finite-difference checks;
* Grad's 13-moment distribution (Grad 1949) integrated over c_z with the Chu
  weights 1 and c_z^2 / 2, and the 13 moments of a Chu distribution.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT, N_USED, N_FOURIER = 64, 128, 16, 9, 12
LAYERS = [(N_IN, N_HID), (N_HID, N_HID), (N_HID, N_HID), (N_HID, N_HID), (N_HID, N_OUT)]


def _offsets():
    w, off = [], 0
    for i, o in LAYERS:
        w.append(off)
        off += i * o
    b = []
    for i, o in LAYERS:
        b.append(off)
        off += o
    return w, b, off


W_OFF, B_OFF, N_PARAMS = _offsets()


def unpack(params):
    """(weights [out][in], biases) views of a flat parameter vector."""
    params = np.asarray(params)
    Ws = [params[W_OFF[l]:W_OFF[l] + i * o].reshape(o, i) for l, (i, o) in enumerate(LAYERS)]
    bs = [params[B_OFF[l]:B_OFF[l] + o] for l, (i, o) in enumerate(LAYERS)]
    return Ws, bs


def bf16(x) -> np.ndarray:
    """Round FP32 values to BF16 (nearest, ties to even), returned as FP32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(x.shape)


def features(q) -> np.ndarray:
    """Features of rows (x/L, y/L, a, b): 2x-1, 2y-1, a, b, then
    sin/cos(k pi x), sin/cos(k pi y) for k = 1..12, then zeros (FP32)."""
    q = np.asarray(q, np.float64)
    f = np.zeros((len(q), N_IN))
    f[:, 0] = 2 * q[:, 0] - 1
    f[:, 1] = 2 * q[:, 1] - 1
    f[:, 2] = q[:, 2]
    f[:, 3] = q[:, 3]
    for k in range(1, N_FOURIER + 1):
        f[:, 4 * k + 0] = np.sin(k * np.pi * q[:, 0])
        f[:, 4 * k + 1] = np.cos(k * np.pi * q[:, 0])
        f[:, 4 * k + 2] = np.sin(k * np.pi * q[:, 1])
        f[:, 4 * k + 3] = np.cos(k * np.pi * q[:, 1])
    return f.astype(np.float32)


def _mm(a, b):
    """FP32 result of a product of FP32 operands (sums taken in FP64)."""
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(np.float32)


def forward(params, X):
    """Kernel-rounded forward of feature rows X.  Returns (O, Ys) with Ys the
    BF16 inputs of each layer (Ys[0] = bf16(X))."""
    Ws, bs = unpack(np.asarray(params, np.float32))
    Y = bf16(X)
    Ys = [Y]
    for l in range(4):
        Z = _mm(Y, bf16(Ws[l]).T) + bs[l]
        Y = bf16(np.tanh(Z.astype(np.float64)).astype(np.float32))
        Ys.append(Y)
    O = _mm(Y, bf16(Ws[4]).T) + bs[4]
    return O, Ys


def loss_grad(params, X, T, w=None):
    """Kernel-rounded loss sum_i sum_c w_c (O_ic - T_ic)^2 and its gradient
    divided by the row count, in the kernels' order of rounding."""
    n = len(X)
    w = np.ones(N_USED, np.float32) if w is None else np.asarray(w, np.float32)
    Ws, bs = unpack(np.asarray(params, np.float32))
    O, Ys = forward(params, X)
    e = np.zeros((n, N_OUT), np.float32)
    e[:, :N_USED] = O[:, :N_USED] - T[:, :N_USED]
    wf = np.zeros(N_OUT, np.float32)
    wf[:N_USED] = w
    loss = float(np.sum(wf * e.astype(np.float64) ** 2))
    dZ = bf16(2.0 * wf * e / np.float32(n))
    g = np.zeros(N_PARAMS, np.float32)
    for l in range(4, -1, -1):
        i, o = LAYERS[l]
        g[W_OFF[l]:W_OFF[l] + i * o] = _mm(dZ.T, Ys[l]).ravel()
        g[B_OFF[l]:B_OFF[l] + o] = dZ.astype(np.float64).sum(0).astype(np.float32)
        if l > 0:
            dY = _mm(dZ, bf16(Ws[l]))
            dZ = bf16(dY * (1.0 - Ys[l] * Ys[l]))
    g[W_OFF[4] + N_USED * N_HID:W_OFF[4] + N_OUT * N_HID] = 0
    g[B_OFF[4] + N_USED:B_OFF[4] + N_OUT] = 0
    return loss, g


def loss_exact(params, X, T, w=None):
    """FP64 loss without any rounding (for finite differences)."""
    w = np.ones(N_USED) if w is None else np.asarray(w, np.float64)
    Ws, bs = unpack(np.asarray(params, np.float64))
    Y = np.asarray(X, np.float64)
    for l in range(4):
        Y = np.tanh(Y @ Ws[l].T + bs[l])
    O = Y @ Ws[4].T + bs[4]
    return float(np.sum(w * (O[:, :N_USED] - T[:, :N_USED]) ** 2))


def grad_exact(params, X, T, w=None):
    """FP64 gradient of loss_exact / n by backpropagation."""
    n = len(X)
    w = np.ones(N_USED) if w is None else np.asarray(w, np.float64)
    Ws, bs = unpack(np.asarray(params, np.float64))
    Ys = [np.asarray(X, np.float64)]
    for l in range(4):
        Ys.append(np.tanh(Ys[-1] @ Ws[l].T + bs[l]))
    O = Ys[-1] @ Ws[4].T + bs[4]
    dZ = np.zeros((n, N_OUT))
    dZ[:, :N_USED] = 2 * w * (O[:, :N_USED] - T[:, :N_USED]) / n
    g = np.zeros(N_PARAMS)
    for l in range(4, -1, -1):
        i, o = LAYERS[l]
        g[W_OFF[l]:W_OFF[l] + i * o] = (dZ.T @ Ys[l]).ravel()
        g[B_OFF[l]:B_OFF[l] + o] = dZ.sum(0)
        if l > 0:
            dZ = (dZ @ Ws[l]) * (1 - Ys[l] ** 2)
    return g


def adam(params, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step in FP32 (bias-corrected, as the update kernel)."""
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    c1, c2 = np.float32(1 - b1 ** t), np.float32(1 - b2 ** t)
    p = params - np.float32(lr) * (m / c1) / (np.sqrt(v / c2) + np.float32(eps))
    return p.astype(np.float32), m, v


# ---------------------------------------------------------------------------
# Grad 13 in the Chu representation
# ---------------------------------------------------------------------------
def velocity_grid(Nv, vmin, dv):
    k = np.arange(Nv * Nv)
    return vmin + (k % Nv) * dv, vmin + (k // Nv) * dv


def grad13_rows(mom, Nv, vmin, dv, R):
    """(g1, g2) rows of Grad's 13-moment distribution for moment rows
    (rho, ux, uy, T, sxx, sxy, syy, qx, qy); negative values set to zero."""
    mom = np.atleast_2d(np.asarray(mom, np.float64))
    vx, vy = velocity_grid(Nv, vmin, dv)
    rho = np.maximum(mom[:, 0:1], 1e-30)
    ux, uy = mom[:, 1:2], mom[:, 2:3]
    th = R * np.maximum(mom[:, 3:4], 1e-6)
    p = rho * th
    sxx, sxy, syy, qx, qy = (mom[:, c:c + 1] for c in range(4, 9))
    szz = -(sxx + syy)
    cx, cy = vx[None, :] - ux, vy[None, :] - uy
    c2 = cx * cx + cy * cy
    M = rho / (2 * np.pi * th) * np.exp(-c2 / (2 * th))
    A = (sxx * cx * cx + 2 * sxy * cx * cy + syy * cy * cy) / (2 * p * th)
    B = (qx * cx + qy * cy) / (p * th)
    g1 = np.maximum(M * (1 + A + szz / (2 * p) + B * (c2 / (5 * th) - 0.8)), 0)
    g2 = np.maximum(0.5 * th * M * (1 + A + 1.5 * szz / p + B * (c2 / (5 * th) - 0.4)), 0)
    return g1, g2


def moments13(g1, g2, Nv, vmin, dv, R):
    """13 moments of Chu rows with the discrete sums of Moments.cpp:66-97:
    rho, ux, uy, T, sigma_xx, sigma_xy, sigma_yy, q_x, q_y."""
    g1 = np.atleast_2d(np.asarray(g1, np.float64))
    g2 = np.atleast_2d(np.asarray(g2, np.float64))
    vx, vy = velocity_grid(Nv, vmin, dv)
    w = dv * dv
    s0 = g1.sum(1)
    rho = s0 * w
    ux = (g1 * vx).sum(1) / s0
    uy = (g1 * vy).sum(1) / s0
    cx, cy = vx[None, :] - ux[:, None], vy[None, :] - uy[:, None]
    e = (cx * cx + cy * cy) * g1 + 2 * g2
    th = e.sum(1) * w / (3 * rho)
    p = rho * th
    out = np.stack([rho, ux, uy, th / R,
                    (cx * cx * g1).sum(1) * w - p, (cx * cy * g1).sum(1) * w,
                    (cy * cy * g1).sum(1) * w - p,
                    0.5 * (cx * e).sum(1) * w, 0.5 * (cy * e).sum(1) * w], axis=1)
    return out
