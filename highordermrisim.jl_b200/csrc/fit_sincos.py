"""Derivation of the sine/cosine polynomial coefficients used by the split
kernel (homs_split.cu) on the reduced argument x in [-pi/4, pi/4]:

    sin(x) ~ x + x^3 (S1 + S2 x^2 + S3 x^4)
    cos(x) ~ 1 + x^2 (C1 + C2 x^2 + C3 x^4 + C4 x^6)

Method: weighted least squares on 4000 Chebyshev nodes, re-weighted 30 times
by the running absolute error (a Lawson-style approximation of the minimax
fit).  Printed are the coefficients rounded to float32 and the worst error of
the float32 evaluation on a dense grid (about 4e-8 for sine, 6.5e-8 for
cosine).  Run: python fit_sincos.py
"""
import numpy as np


def fit():
    a = np.pi / 4
    n = 4000
    x = a * np.cos(np.pi * (np.arange(n) + 0.5) / n)
    x2 = x * x

    def lsq(target, w, deg):
        A = np.stack([x2 ** i for i in range(deg)], axis=1)
        return np.linalg.lstsq(A * w[:, None], target * w, rcond=None)[0]

    w = np.ones(n)
    ts = (np.sin(x) - x) / x ** 3
    for _ in range(30):
        cs = lsq(ts, w, 3)
        err = x + x ** 3 * (np.stack([x2 ** i for i in range(3)], 1) @ cs) - np.sin(x)
        w = w * (1 + np.abs(err) / np.abs(err).max())
    w = np.ones(n)
    tc = (np.cos(x) - 1) / x2
    for _ in range(30):
        cc = lsq(tc, w, 4)
        errc = 1 + x2 * (np.stack([x2 ** i for i in range(4)], 1) @ cc) - np.cos(x)
        w = w * (1 + np.abs(errc) / np.abs(errc).max())
    return [np.float32(c) for c in cs], [np.float32(c) for c in cc]


if __name__ == "__main__":
    s, c = fit()
    print("S1..S3 =", [repr(float(v)) for v in s])
    print("C1..C4 =", [repr(float(v)) for v in c])
