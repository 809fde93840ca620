"""CPU oracle of the learned corrector (test infrastructure only).

The network has no counterpart in the reference; this is a NumPy restatement
of its mathematics, written from the definitions: three periodic 3^3
convolutions (4 -> 32 -> 32 -> 2 channels), GELU(z) = z Phi(z) between them, a
mean-square loss against (psi_f - psi_c) / tau, and the parameter gradients by
the chain rule (the data gradient of a periodic convolution is the
convolution with spatially reflected, channel-transposed weights).

`bf16=True` rounds at the same places the device path does (features, weights,
hidden activations and the back-propagated data gradients are BF16; sums are
FP64 here, FP32 on the device), so the device gradients can be compared at
round-off level.  Arrays are [z][y][x][channel]; parameter layout
w[o][ci][co], o = (dz+1)*9 + (dy+1)*3 + (dx+1).
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

DIMS = [(4, 32), (32, 32), (32, 2)]
OFFS = [((o // 9) - 1, ((o // 3) % 3) - 1, (o % 3) - 1) for o in range(27)]  # (dz, dy, dx)


def bf16(a):
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    """Flat parameter vector -> [(w [27][ci][co], b [co])] per layer."""
    out, k = [], 0
    for ci, co in DIMS:
        n = 27 * ci * co
        w = np.asarray(params[k:k + n], np.float64).reshape(27, ci, co)
        k += n
        b = np.asarray(params[k:k + co], np.float64)
        k += co
        out.append((w, b))
    return out


def shift(a, o):
    """a[z + dz][y + dy][x + dx] (periodic)."""
    dz, dy, dx = OFFS[o]
    return np.roll(a, shift=(-dz, -dy, -dx), axis=(0, 1, 2))


def unshift(a, o):
    dz, dy, dx = OFFS[o]
    return np.roll(a, shift=(dz, dy, dx), axis=(0, 1, 2))


def conv(a, w, b):
    z = np.zeros(a.shape[:3] + (w.shape[2],))
    for o in range(27):
        z += shift(a, o) @ w[o]
    return z + b


def conv_t(dz, w):
    """Data gradient of conv: sum_o unshift(dz @ w[o]^T)."""
    da = np.zeros(dz.shape[:3] + (w.shape[1],))
    for o in range(27):
        da += unshift(dz @ w[o].T, o)
    return da


def wgrad(a, dz):
    ci, co = a.shape[3], dz.shape[3]
    dw = np.zeros((27, ci, co))
    A = None
    D = dz.reshape(-1, co)
    for o in range(27):
        A = shift(a, o).reshape(-1, ci)
        dw[o] = A.T @ D
    return dw, D.sum(axis=0)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def features(psi_c, V_c, v_scale):
    """[N,N,N,4]: Re psi, Im psi, V / v_scale, |psi|^2 - 1 (FP32 inputs)."""
    p = np.asarray(psi_c, np.complex64)
    v = np.asarray(V_c, np.float32)
    f = np.stack([p.real, p.imag, (v * np.float32(1.0 / v_scale)),
                  p.real * p.real + p.imag * p.imag - np.float32(1.0)], axis=-1)
    return f.astype(np.float64)


def forward(params, psi_c, V_c, v_scale, bf=True):
    r = (lambda x: bf16(x)) if bf else (lambda x: x)
    L = unpack(params)
    x0 = r(features(psi_c, V_c, v_scale))
    ws = [(r(w), b) for w, b in L]
    z1 = conv(x0, *ws[0])
    a1 = r(gelu(z1))
    z2 = conv(a1, *ws[1])
    a2 = r(gelu(z2))
    y = conv(a2, *ws[2])
    return dict(x0=x0, z1=z1, a1=a1, z2=z2, a2=a2, y=y, ws=ws)


def loss_and_grads(params, psi_c, V_c, psi_f, v_scale, tau, bf=True):
    """Mean-square loss over sites and the 2 output channels, and its gradient
    with respect to the parameters (flat, in the parameter layout)."""
    r = (lambda x: bf16(x)) if bf else (lambda x: x)
    st = forward(params, psi_c, V_c, v_scale, bf)
    pf = np.asarray(psi_f, np.complex64)
    pc = np.asarray(psi_c, np.complex64)
    d = (pf - pc) * np.float32(1.0 / tau)
    T = np.stack([d.real, d.imag], axis=-1).astype(np.float64)
    n = T.size
    diff = st["y"] - T
    loss = float(np.sum(diff * diff) / n)
    dy = 2.0 * diff / n
    (w1, _), (w2, _), (w3, _) = st["ws"]
    g3w, g3b = wgrad(st["a2"], dy)
    da2 = conv_t(r(dy), w3)
    dz2 = da2 * gelu_grad(st["z2"])
    g2w, g2b = wgrad(st["a1"], dz2)
    da1 = conv_t(r(dz2), w2)
    dz1 = da1 * gelu_grad(st["z1"])
    g1w, g1b = wgrad(st["x0"], dz1)
    grads = np.concatenate([g1w.ravel(), g1b, g2w.ravel(), g2b, g3w.ravel(), g3b])
    return loss, grads, st["y"]


def nparams():
    return sum(27 * ci * co + co for ci, co in DIMS)
