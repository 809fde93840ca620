"""Fit the polynomials of the FP32 kick's sin/cos (qx_kernels.cuh, cis_kick).

The kick phase is reduced in FP64 to r in [-pi/4, pi/4] plus a quadrant, so
sin and cos are needed on that interval only:
    sin r ~ r + r^3 (s1 + r^2 (s2 + r^2 s3))
    cos r ~ 1 + r^2 (c1 + r^2 (c2 + r^2 (c3 + r^2 c4)))
The coefficients are a weighted least-squares fit on Chebyshev nodes (close to
the minimax polynomial of the same degree), computed in float64, then rounded
to float32 and checked by evaluating the polynomials in float32 arithmetic
against numpy's float64 sin/cos.  Run: python fit_kick_poly.py
"""
import numpy as np


def fit():
    n = 4000
    h = np.pi / 4
    x = h * np.cos(np.pi * (np.arange(n) + 0.5) / n)  # Chebyshev nodes on [-h, h]
    x = x[x != 0]
    # sin: (sin x - x) / x^3 as a polynomial in x^2 (relative-error weighting)
    A = np.stack([x**0, x**2, x**4], axis=1)
    s, *_ = np.linalg.lstsq(A, (np.sin(x) - x) / x**3, rcond=None)
    # cos: (cos x - 1) / x^2 as a polynomial in x^2
    B = np.stack([x**0, x**2, x**4, x**6], axis=1)
    c, *_ = np.linalg.lstsq(B, (np.cos(x) - 1) / x**2, rcond=None)
    return s.astype(np.float32), c.astype(np.float32)


def eval_f32(r, s, c):
    r = np.float32(r)
    r2 = r * r
    sp = np.float32(s[0]) + r2 * (np.float32(s[1]) + r2 * np.float32(s[2]))
    sn = r + (r * r2) * sp
    cp = np.float32(c[0]) + r2 * (np.float32(c[1]) + r2 * (np.float32(c[2]) + r2 * np.float32(c[3])))
    cs = np.float32(1) + r2 * cp
    return sn, cs


if __name__ == "__main__":
    s, c = fit()
    r = np.linspace(-np.pi / 4, np.pi / 4, 200001).astype(np.float32)
    sn, cs = eval_f32(r, s, c)
    rd = r.astype(np.float64)
    print("sin coefficients", [float.hex(float(v)) for v in s], s.tolist())
    print("cos coefficients", [float.hex(float(v)) for v in c], c.tolist())
    print("max |sin err|", np.max(np.abs(sn - np.sin(rd))), "max |cos err|", np.max(np.abs(cs - np.cos(rd))))
