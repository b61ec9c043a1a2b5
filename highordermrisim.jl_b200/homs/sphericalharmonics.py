"""Real solid-harmonic basis functions, unnormalised, in metres
(``basisfunc_spha``, src/sphericalharmonics/basisfunction.jl:24-120).

Terms are 1-based as in the reference: 1 is the constant, 2-4 the first
order (x, y, z), 5-9 the second, 10-16 the third (the sixteen terms the
simulation uses, h0..h15), 17-25 the fourth and 26-36 the fifth order.  Host
NumPy: the engine evaluates terms 1-16 on the device itself.
"""
from __future__ import annotations

import numpy as np

from .model import ArgumentError

__all__ = ["basisfunc_spha", "NTERMS_SPHA"]

NTERMS_SPHA = 36


def _term(k: int, x, y, z):
    r2 = x * x + y * y + z * z
    if k == 1:
        return np.ones_like(x)
    if k == 2:
        return x
    if k == 3:
        return y
    if k == 4:
        return z
    if k == 5:
        return x * y
    if k == 6:
        return z * y
    if k == 7:
        return 3 * z ** 2 - r2
    if k == 8:
        return x * z
    if k == 9:
        return x ** 2 - y ** 2
    if k == 10:
        return 3 * y * x ** 2 - y ** 3
    if k == 11:
        return x * z * y
    if k == 12:
        return (5 * z ** 2 - r2) * y
    if k == 13:
        return 5 * z ** 3 - 3 * z * r2
    if k == 14:
        return (5 * z ** 2 - r2) * x
    if k == 15:
        return x ** 2 * z - y ** 2 * z
    if k == 16:
        return x ** 3 - 3 * x * y ** 2
    if k == 17:
        return (x * y) * (x ** 2 - y ** 2)
    if k == 18:
        return (y * z) * (3 * x ** 2 - y ** 2)
    if k == 19:
        return (x * y) * (7 * z ** 2 - r2)
    if k == 20:
        return y * (7 * z ** 3 - 3 * z * r2)
    if k == 21:
        return 35 * z ** 4 - 30 * z ** 2 * r2 + 3 * r2 ** 2
    if k == 22:
        return x * (7 * z ** 3 - 3 * z * r2)
    if k == 23:
        return (x ** 2 - y ** 2) * (7 * z ** 2 - r2)
    if k == 24:
        return x * (x ** 2 - 3 * y ** 2) * z
    if k == 25:
        return x ** 2 * (x ** 2 - 3 * y ** 2) - y ** 2 * (3 * x ** 2 - y ** 2)
    if k == 26:
        return y * (5 * x ** 4 - 10 * x ** 2 * y ** 2 + y ** 4)
    if k == 27:
        return x * y * z * (x ** 2 - y ** 2)
    if k == 28:
        return y * (r2 - 9 * z ** 2) * (y ** 2 - 3 * x ** 2)
    if k == 29:
        return x * y * z * (3 * z ** 2 - r2)
    if k == 30:
        return y * (r2 ** 2 - 14 * r2 * z ** 2 + 21 * z ** 4)
    if k == 31:
        return 63 * z ** 5 - 70 * z ** 3 * r2 + 15 * z * r2 ** 2
    if k == 32:
        return x * (r2 ** 2 - 14 * r2 * z ** 2 + 21 * z ** 4)
    if k == 33:
        return z * (3 * z ** 2 - r2) * (x ** 2 - y ** 2)
    if k == 34:
        return x * (r2 - 9 * z ** 2) * (3 * y ** 2 - x ** 2)
    if k == 35:
        return z * (x ** 4 - 6 * x ** 2 * y ** 2 + y ** 4)
    if k == 36:
        return x ** 5 - 10 * x ** 3 * y ** 2 + 5 * x * y ** 4
    raise ArgumentError("Basis function undefined.")


def basisfunc_spha(x, y, z, terms):
    """(nSample, nTerm) basis values for the 1-based ``terms`` (a list, or one
    int for a single column returned as a vector), in the coordinates' float
    type."""
    x, y, z = (np.asarray(v) for v in (x, y, z))
    if not (x.shape == y.shape == z.shape and x.ndim == 1):
        raise ArgumentError("x, y and z must be vectors of one length.")
    dt = np.result_type(x.dtype, y.dtype, z.dtype, np.float32)
    x, y, z = (v.astype(dt) for v in (x, y, z))
    if isinstance(terms, (int, np.integer)):
        return _term(int(terms), x, y, z).astype(dt)
    out = np.zeros((x.shape[0], len(terms)), dtype=dt)
    for i, k in enumerate(terms):
        out[:, i] = _term(int(k), x, y, z)
    return out
