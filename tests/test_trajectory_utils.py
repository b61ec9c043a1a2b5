"""Measured-trajectory utilities, on the cases of the reference's
test/unit/test_trajectory_utils.jl (Float32 and Float64)."""
import numpy as np
import pytest

from homs import ArgumentError, InterpTrajTime, grad2traj, traj2grad


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_reference_cases(T):
    dt = T(0.25)
    values = np.arange(12, dtype=T).reshape(3, 4).T  # Julia reshape(T.(0:11), 4, 3)
    assert np.array_equal(traj2grad(values, dt), np.diff(values, axis=0) / dt)
    expected = np.vstack([np.zeros((1, 3), T), np.cumsum((values[:3] + values[1:]) * (dt / T(2)), axis=0)])
    got = grad2traj(values, dt)
    assert got.dtype == T and np.array_equal(got, expected)
    assert np.array_equal(grad2traj(values.T, dt, dim=2), expected.T)
    assert grad2traj(np.zeros((0, 3), T), dt).shape == (0, 3)
    assert traj2grad(np.zeros((0, 3), T), dt).shape == (0, 3)
    assert traj2grad(np.ones((1, 3), T), dt).shape == (0, 3)
    for op in (grad2traj, traj2grad):
        for bad in (0, -1, np.inf, np.nan):
            with pytest.raises(ArgumentError):
                op(values, bad)
        for dim in (0, 3):
            with pytest.raises(ArgumentError):
                op(values, dt, dim=dim)
    times = np.arange(4, dtype=np.float64) * float(dt)
    interp = InterpTrajTime(values, dt, 0.0, times)
    assert np.allclose(interp, values) and interp.dtype == T
    assert np.allclose(InterpTrajTime(values, dt, 0.0), values)
    assert InterpTrajTime(np.zeros((4, 0), T), dt, 0.0, times).shape == (4, 0)
    assert InterpTrajTime(values, dt, 0.0, np.zeros(0)).shape == (0, 3)
    for bad in (0, -1, np.inf, np.nan):
        with pytest.raises(ArgumentError):
            InterpTrajTime(values, bad, 0.0, times)
    with pytest.raises(ArgumentError):
        InterpTrajTime(values, dt, np.inf, times)
    with pytest.raises(ArgumentError):
        InterpTrajTime(values, dt, 0.0, [0.0, np.nan])
    shots = np.stack([values, 2 * values])
    sampled = InterpTrajTime(shots, dt, [0.0, 0.0], np.tile(times, (2, 1)))
    assert np.allclose(sampled, shots) and sampled.dtype == T


def test_interpolation_between_knots_delay_and_outside():
    dt = 1e-3
    t = np.arange(50) * dt
    y = np.stack([np.sin(2 * np.pi * 7 * t), 3 * t - 0.01], axis=1)
    q = np.linspace(-2e-3, 52e-3, 400)
    out = InterpTrajTime(y, dt, 0.0, q)
    inside = (q >= 0) & (q <= t[-1])
    assert np.all(out[~inside] == 0)
    assert np.allclose(out[inside, 1], 3 * q[inside] - 0.01, atol=1e-12)  # Akima reproduces lines
    assert np.max(np.abs(out[inside, 0] - np.sin(2 * np.pi * 7 * q[inside]))) < 2e-3
    shifted = InterpTrajTime(y, dt, 5 * dt, t[:40])  # knots moved 5 samples earlier
    assert np.allclose(shifted[:, 0], y[5:45, 0])
    lin = InterpTrajTime(y, dt, 0.0, q, intermode="linear")
    assert np.allclose(lin[inside, 1], 3 * q[inside] - 0.01, atol=1e-12)
