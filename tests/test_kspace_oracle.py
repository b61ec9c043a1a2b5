"""Encoding export oracle (grad2kspace, src/datatypes/HO_Sequence.jl:257-287)
against closed forms and the reference's own get_kspace tests."""
import numpy as np
import pytest

from homs.model import GAMMA, HO_DiscreteSequence, rf_events
from homs import workloads as W
from oracle import oracle as orc


def _seq(nt, dt=1e-5, gx=0.0, gy=0.0, gz=0.0, h=None, b1=None, excitation=None):
    t = np.arange(nt) * dt
    return HO_DiscreteSequence(t, dt=np.full(nt - 1, dt), gx=np.broadcast_to(gx, (nt,)).copy(),
                               gy=np.broadcast_to(gy, (nt,)).copy(), gz=np.broadcast_to(gz, (nt,)).copy(),
                               b1=b1, excitation=excitation, h=h)


def test_cumtrapz_is_the_trapezoid_prefix():
    dt = np.array([0.5, 0.25, 1.0])
    x = np.array([1.0, 3.0, -1.0, 2.0])
    assert np.allclose(orc.cumtrapz_np(dt, x), np.cumsum([0.5 * 2.0, 0.25 * 1.0, 1.0 * 0.5]), rtol=0, atol=0)


def test_kfoldperm_breaks_start_parts():
    assert orc.kfoldperm_parts(10, []) == [(0, 10)]
    assert orc.kfoldperm_parts(10, [4, 8]) == [(0, 3), (3, 7), (7, 10)]
    assert orc.kfoldperm_parts(10, [1, 4]) == [(0, 3), (3, 10)]  # a break at 1 opens no part


def test_constant_gradient_is_gamma_g_t():
    g = 2e-3
    seq = _seq(101, gx=g, gz=-g)
    k, _ = orc.grad2kspace_np(seq, [], [])
    t_end = np.asarray(seq.t[1:])
    assert np.allclose(k[:, 0], GAMMA * g * t_end, rtol=1e-13)
    assert np.allclose(k[:, 2], -GAMMA * g * t_end, rtol=1e-13)
    assert np.all(k[:, 1] == 0) and np.all(k[:, 3:] == 0)


def test_measured_is_twice_nominal_when_the_field_is_twice_the_gradient():
    # test/unit/test_spatial_plots.jl:12-17: GR_dfc[2:4] = 2 GR => measured[:, 2:4] = 2 nominal
    rng = np.random.default_rng(3)
    nt = 300
    g = rng.standard_normal((3, nt)) * 1e-3
    h = np.zeros((16, nt))
    h[1:4] = 2 * g
    seq = _seq(nt, gx=g[0], gy=g[1], gz=g[2], h=h)
    k, _ = orc.grad2kspace_np(seq, [100, 200], [0, -1])
    assert np.allclose(k[:, 4:7], 2 * k[:, 0:3], rtol=1e-13, atol=0)


def test_zero_waveforms_give_zero_adc_encoding():
    # test/unit/test_koma_compatibility.jl:46-52
    w, _, _, _ = W.compatibility_sequence()
    k, kq = orc.grad2kspace_np(w, *rf_events(w), q_times=np.asarray(w.t)[np.asarray(w.adc)])
    assert k.shape[1] == 19 and kq.shape == (5, 19)
    assert np.all(kq == 0)


def test_excitation_restarts_and_refocusing_negates():
    nt, g = 41, 1e-3
    seq = _seq(nt, gx=g)
    step = GAMMA * g * 1e-5
    k, _ = orc.grad2kspace_np(seq, [10, 25], [0, -1])
    assert np.isclose(k[9, 0], 10 * step, rtol=1e-13)
    assert np.isclose(k[10, 0], step, rtol=1e-13)          # restarted
    assert np.isclose(k[24, 0], 15 * step, rtol=1e-13)
    assert np.isclose(k[25, 0], step - 15 * step, rtol=1e-12)  # negated, then continued
    k2, _ = orc.grad2kspace_np(seq, [10, 25], [1, 1])    # skipped pulses
    assert np.allclose(k2[:, 0], GAMMA * g * np.asarray(seq.t[1:]), rtol=1e-12)


def test_adc_interpolation_hits_node_values_and_zero_outside():
    seq = _seq(21, gx=1e-3)
    k, kq = orc.grad2kspace_np(seq, [], [], q_times=[-1.0, 0.0, 1e-5, 1.5e-5, 2e-4, 3e-4])
    assert kq[0, 0] == 0 and kq[1, 0] == 0 and kq[5, 0] == 0  # before the first knot / after the last
    assert kq[2, 0] == k[0, 0] and kq[4, 0] == k[-1, 0]
    assert np.isclose(kq[3, 0], 0.5 * (k[0, 0] + k[1, 0]), rtol=1e-14)


def test_rf_events_of_the_workloads():
    assert rf_events(W.config(0).seq) == ([1], [0])
    starts, signs = rf_events(W.config(1).seq)
    assert len(starts) == 4 and signs == [0, 0, 0, 0]
    nt = 60
    b1 = np.zeros(nt, np.complex128)
    exc = np.zeros(nt - 1, bool)
    b1[10:20] = 1.0 / (2 * GAMMA * 1e-4)  # 180 degrees over 10 x 1e-5 s
    exc[10:20] = True
    seq = _seq(nt, b1=b1, excitation=exc)
    assert rf_events(seq) == ([15], [-1])
    assert rf_events(seq, skip_rf=[True]) == ([15], [1])
    with pytest.raises(ValueError):
        rf_events(seq, skip_rf=[True, False])
