"""CPU oracle of the learned LBGK closure — TEST INFRASTRUCTURE ONLY.

Imported by tests/ only; the product path (asl_b200) never calls it. The
closure is an extension of this project (ASL's LBGKTurbulence,
src/num/aslLBGK.cxx:298-355, has a fixed limiter instead), so there is no
reference source to follow: this file restates, in float64 numpy, the
definitions the CUDA code implements, independently of that code:

* features(rho, u, Pi): the nine inputs of the network from density,
  velocity and the non-equilibrium stress Pi_ab = sum_i w_i c_ia c_ib
  (f_i - f_eq,i) (ASL normalisation);
* moments_pneq(f, q, ...): rho, u and Pi of a cell from its incoming
  populations, with f_eq in ASL's form (rho + 3 c.m + 4.5 (c.m)^2/rho - 1.5 m.m/rho);
* forward / backward of the 9 -> 64 -> 64 -> 1 network, the loss
  mean((out_scale softplus(y) - t)^2), and one Adam step;
* infer_bf16: the inference path with BF16-rounded inputs, weights and
  hidden activations (what the tensor-core kernel computes).
"""
from __future__ import annotations

import numpy as np

N_IN, N_H = 9, 64


def bf16(a):
    """Round float64/float32 values to the nearest bfloat16 (ties to even)."""
    a32 = np.asarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def features(rho, ux, uy, uz, P):
    """Nine invariants per cell; P = (P00, P11, P22, P01, P12, P02), arrays."""
    ir = 1.0 / rho
    a, b, c, d, e, g = (p * ir for p in P)
    tr = a + b + c
    t3 = tr / 3.0
    da, db, dc = a - t3, b - t3, c - t3
    off2 = d * d + e * e + g * g
    n2 = a * a + b * b + c * c + 2 * off2
    dn2 = da * da + db * db + dc * dc + 2 * off2
    det = a * (b * c - e * e) - d * (d * c - e * g) + g * (d * e - b * g)
    ddet = da * (db * dc - e * e) - d * (d * dc - e * g) + g * (d * e - db * g)
    return np.stack([tr, np.sqrt(n2), np.sqrt(dn2), np.cbrt(3 * ddet), np.cbrt(det), np.log(np.sqrt(dn2) + 1e-12),
                     np.sqrt(a * a + b * b + c * c), np.sqrt(2 * off2), np.sqrt(ux * ux + uy * uy + uz * uz)])


def moments_pneq(f, c, w, compressible=True):
    """f: (Q, ...) incoming populations; c: (Q, 3) velocities; w: (Q,) weights."""
    rho = np.tensordot(w, f, axes=(0, 0))
    m = np.stack([np.tensordot(w * c[:, a], f, axes=(0, 0)) for a in range(3)])
    cm = np.tensordot(c, m, axes=(1, 0))  # (Q, ...)
    mm = (m * m).sum(0)
    if compressible:
        feq = rho + 3 * cm + 4.5 * cm * cm / rho - 1.5 * mm / rho
        u = m / rho
    else:
        feq = rho + 3 * cm + 4.5 * cm * cm - 1.5 * mm
        u = m
    d = f - feq
    idx = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    P = [np.tensordot(w * c[:, a] * c[:, b], d, axes=(0, 0)) for a, b in idx]
    return rho, u, P


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    W1 = p[o:o + N_H * N_IN].reshape(N_H, N_IN); o += N_H * N_IN
    b1 = p[o:o + N_H]; o += N_H
    W2 = p[o:o + N_H * N_H].reshape(N_H, N_H); o += N_H * N_H
    b2 = p[o:o + N_H]; o += N_H
    w3 = p[o:o + N_H]; o += N_H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def param_count():
    return N_H * N_IN + N_H + N_H * N_H + N_H + N_H + 1


def softplus(y):
    return np.where(y > 20, y, np.log1p(np.exp(np.minimum(y, 20))))


def forward(params, x, norm):
    """x: (9, n). Returns Cs^2 (n,) and the activations."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    xn = (x - norm[:N_IN, None]) * norm[N_IN:, None]
    a1 = W1 @ xn + b1[:, None]
    h1 = np.maximum(a1, 0)
    a2 = W2 @ h1 + b2[:, None]
    h2 = np.maximum(a2, 0)
    y = w3 @ h2 + b3
    return y, (xn, a1, h1, a2, h2)


def loss_and_grad(params, x, t, norm, out_scale):
    """Sum of squared errors and the gradient of the MEAN squared error."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    y, (xn, a1, h1, a2, h2) = forward(params, x, norm)
    n = x.shape[1]
    e = out_scale * softplus(y) - t
    dy = 2 * e * out_scale / (1 + np.exp(-y)) / n
    gw3 = h2 @ dy
    gb3 = dy.sum()
    dh2 = np.outer(w3, dy) * (a2 > 0)
    gW2 = dh2 @ h1.T
    gb2 = dh2.sum(1)
    dh1 = (W2.T @ dh2) * (a1 > 0)
    gW1 = dh1 @ xn.T
    gb1 = dh1.sum(1)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return float((e * e).sum()), g


def adam(params, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    p = params - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v


def infer_bf16(params, x, norm, out_scale):
    """Cs^2 as the tensor-core inference computes it: BF16 inputs, weights and
    first-layer activations, FP32-exact accumulation, BF16 output weights."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    xn = bf16((x - norm[:N_IN, None]) * norm[N_IN:, None])
    h1 = bf16(np.maximum(bf16(W1) @ xn + b1[:, None], 0))
    h2 = np.maximum(bf16(W2) @ h1 + b2[:, None], 0)
    y = bf16(w3) @ h2 + b3
    return out_scale * softplus(y)
