"""Measured-trajectory utilities of the reference's input path.

``grad2traj`` / ``traj2grad`` follow src/utils/conversion.jl (trapezoidal
cumulative integration and its finite-difference counterpart), and
``InterpTrajTime`` follows src/utils/InterpTraj.jl:33-104 (resampling a
field-camera trajectory onto simulation times, knots dt * (0:n-1) - delTime,
zero outside them).  These prepare field coefficients on the host before a
simulation; they are not on the GPU path.

The reference interpolates with Interpolations.jl's Akima monotonic
interpolation, a third-party package that is not vendored.  Here the
interpolant is Akima's (1970) method, tangents

    t_i = (|m_{i+1} - m_i| m_{i-1} + |m_{i-1} - m_{i-2}| m_i)
          / (|m_{i+1} - m_i| + |m_{i-1} - m_{i-2}|)

(the mean of m_{i-1}, m_i where the weights vanish), slopes beyond the ends
extended linearly as in Akima's paper, and cubic Hermite segments.  It
passes through every knot, as the reference's tests require; between knots
near the ends it may differ from Interpolations.jl's boundary treatment.
"""
from __future__ import annotations

import math

import numpy as np

from .model import ArgumentError

_INTERP_MODES = ("akima", "linear")


def _check_dt(dt):
    if not (isinstance(dt, (int, float, np.integer, np.floating)) and math.isfinite(float(dt)) and float(dt) > 0):
        raise ArgumentError("The sample interval must be finite and positive.")


def _check_axis(x: np.ndarray, dt, dim: int):
    _check_dt(dt)
    if not 1 <= dim <= x.ndim:
        raise ArgumentError("dim must identify an input array dimension.")


def grad2traj(x, dt, dim: int = 1) -> np.ndarray:
    """Trapezoidal cumulative integral along axis ``dim`` (1-based, as in
    Julia): zero first sample, then cumsum((x[1:end-1] + x[2:end]) .* (dt/2))
    (src/utils/conversion.jl:30-52).  No gamma or unit conversion."""
    x = np.asarray(x)
    _check_axis(x, dt, dim)
    ax = dim - 1
    n = x.shape[ax]
    if n == 0:
        return np.empty(x.shape, dtype=np.result_type(x.dtype, np.float32))
    half = x.dtype.type(dt / 2) if np.issubdtype(x.dtype, np.floating) else dt / 2
    lo = np.take(x, np.arange(n - 1), axis=ax)
    hi = np.take(x, np.arange(1, n), axis=ax)
    cs = np.cumsum((lo + hi) * half, axis=ax)
    zshape = list(x.shape)
    zshape[ax] = 1
    return np.concatenate([np.zeros(zshape, dtype=cs.dtype), cs], axis=ax)


def traj2grad(x, dt, dim: int = 1) -> np.ndarray:
    """Consecutive differences along ``dim`` divided by dt
    (src/utils/conversion.jl:76-89): one value per interval."""
    x = np.asarray(x)
    _check_axis(x, dt, dim)
    ax = dim - 1
    n = x.shape[ax]
    if n == 0:
        return np.empty(x.shape, dtype=np.result_type(x.dtype, np.float32))
    step = x.dtype.type(dt) if np.issubdtype(x.dtype, np.floating) else dt
    return np.diff(x, axis=ax) / step


def _akima_tangents(t: np.ndarray, y: np.ndarray) -> np.ndarray:
    m = np.diff(y) / np.diff(t)
    n = y.shape[0]
    if n == 2:
        return np.array([m[0], m[0]])
    # Two slopes beyond each end, extended linearly (Akima 1970).
    ext = np.empty(n + 3)
    ext[2:n + 1] = m
    ext[1] = 2 * m[0] - m[1]
    ext[0] = 2 * ext[1] - m[0]
    ext[n + 1] = 2 * m[-1] - m[-2]
    ext[n + 2] = 2 * ext[n + 1] - m[-1]
    mm2, mm1, m0, mp1 = ext[0:n], ext[1:n + 1], ext[2:n + 2], ext[3:n + 3]
    w1, w2 = np.abs(mp1 - m0), np.abs(mm1 - mm2)
    den = w1 + w2
    flat = den == 0
    return np.where(flat, 0.5 * (mm1 + m0), (w1 * mm1 + w2 * m0) / np.where(flat, 1.0, den))


def _interp_column(t: np.ndarray, y: np.ndarray, q: np.ndarray, mode: str) -> np.ndarray:
    out = np.zeros(q.shape[0])
    inside = (q >= t[0]) & (q <= t[-1])
    if not inside.any():
        return out
    qi = q[inside]
    k = np.clip(np.searchsorted(t, qi, side="right") - 1, 0, t.shape[0] - 2)
    h = t[k + 1] - t[k]
    s = (qi - t[k]) / h
    if mode == "linear":
        out[inside] = y[k] + s * (y[k + 1] - y[k])
        return out
    tan = _akima_tangents(t, y)
    s2, s3 = s * s, s * s * s
    h00, h10, h01, h11 = 2 * s3 - 3 * s2 + 1, s3 - 2 * s2 + s, -2 * s3 + 3 * s2, s3 - s2
    out[inside] = h00 * y[k] + h10 * h * tan[k] + h01 * y[k + 1] + h11 * h * tan[k + 1]
    return out


def InterpTrajTime(traj, dt, delTime, datatime=None, intermode: str = "akima") -> np.ndarray:  # noqa: N802
    """Resample a measured trajectory onto output times.

    ``traj``: (nSample, nTerm), or (nShot, nSample, nTerm) with one delay and
    one row of output times per shot.  Input knots are dt * (0:nSample-1) -
    delTime; values outside them are 0; the result keeps the trajectory's
    element type (src/utils/InterpTraj.jl:33-104).  Without ``datatime`` the
    output times are the input sample times dt * (0:nSample-1)."""
    if intermode not in _INTERP_MODES:
        raise ArgumentError(f"intermode must be one of {_INTERP_MODES}.")
    traj = np.asarray(traj)
    if traj.ndim == 3:
        dels = np.asarray(delTime, dtype=np.float64).reshape(-1)
        times = np.asarray(datatime, dtype=np.float64)
        if dels.shape[0] != traj.shape[0] or times.ndim != 2 or times.shape[0] != traj.shape[0]:
            raise ArgumentError("Number of shots in trajectory, delTime and datatime must match.")
        _check_dt(dt)
        out = np.empty((traj.shape[0], times.shape[1], traj.shape[2]), dtype=traj.dtype)
        for s in range(traj.shape[0]):
            out[s] = InterpTrajTime(traj[s], dt, dels[s], times[s], intermode)
        return out
    if traj.ndim != 2:
        raise ArgumentError("traj must be (nSample, nTerm) or (nShot, nSample, nTerm).")
    _check_dt(dt)
    n, nterm = traj.shape
    if n < 2:
        raise ArgumentError("Trajectory interpolation needs at least two input samples.")
    if not math.isfinite(float(delTime)):
        raise ArgumentError("The trajectory delay must be finite.")
    if datatime is None:
        datatime = float(dt) * np.arange(n)
    q = np.asarray(datatime, dtype=np.float64).reshape(-1)
    if not np.all(np.isfinite(q)):
        raise ArgumentError("Output sample times must be finite.")
    knots = float(dt) * np.arange(n) - float(delTime)
    out = np.empty((q.shape[0], nterm), dtype=traj.dtype)
    for j in range(nterm):
        out[:, j] = _interp_column(knots, traj[:, j].astype(np.float64), q, intermode)
    return out
