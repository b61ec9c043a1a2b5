"""Event-level sequences and their discretisation, on the CPU.

The sampling behaviour the reference fixes (test/unit/test_koma_compatibility.jl:11-53)
is checked exactly as it states it; the reference's known answers for the legacy
simulation path (:55-136) are checked through the FP64 oracle on the discretised
sequences; closed-form properties (exact gradient areas, step limits, ADC times,
RF support and area) are checked on seeded sequences with jumps, shaped pulses and
measured fields."""
import math

import numpy as np
import pytest

import homs
from homs import workloads as W
from homs.model import GAMMA, ArgumentError, BlochHighOrder, DimensionMismatch, count_block_adc, get_sim_ranges
from homs.sequence import (ADC, RF, Grad, HO_Sequence, MaxStepSizeRule, Sequence, discretize,
                           get_adc_phase_compensation, get_adc_sampling_times, get_block_start_times, rf_pulses)


def _trapz(dt, x):
    x = np.asarray(x)
    return float(np.sum((x[1:] + x[:-1]) / 2 * dt))


# -- the reference's sampling tests (test_koma_compatibility.jl:11-53) ---------

def test_parameterized_grad_inputs():
    gradients = [[Grad(float(i), 1e-3)] for i in range(1, 5)]
    hoseq = HO_Sequence(gradients)
    assert [g.A for g in hoseq.SEQ.GR[:, 0]] == [2.0, 3.0, 4.0]
    assert hoseq.GR_dfc.shape == (16, 1)
    assert isinstance(HO_Sequence(hoseq.SEQ, gradients), HO_Sequence)


def test_high_order_only_sampling_keeps_field_jumps():
    jump = HO_Sequence([[Grad(1e-6, 1e-3), Grad(-2e-6, 1e-3)]])
    original = jump.SEQ.DUR.copy()
    sampled = discretize(jump, sampling_params={"Δt": 2e-4})
    assert np.array_equal(jump.SEQ.DUR, original)
    assert math.isclose(sampled.t[-1], 2e-3, rel_tol=1e-12)
    assert np.all(sampled.dt >= 0)
    assert np.any(sampled.dt == 0)
    assert abs(_trapz(sampled.dt, sampled.h[0]) - (-1e-9)) <= 1e-20
    assert sampled.t.shape[0] == sampled.dt.shape[0] + 1
    assert sampled.excitation.shape[0] == sampled.dt.shape[0]
    assert sampled.h.shape == (16, sampled.t.shape[0])
    v = sampled.view(0, 2)
    assert len(v) == 2 and v.h[0].shape[0] == 3
    assert np.array_equal(v.h[0], sampled.h[0][:3])


def test_adc_ownership_and_native_times():
    seq = W.compatibility_events()
    hoseq = HO_Sequence(seq)
    sampled = discretize(hoseq)
    parts, _ = get_sim_ranges(sampled, max_block_length=1)
    assert sum(count_block_adc(sampled.adc, parts)) == 5
    native = get_adc_sampling_times(seq)
    assert np.allclose(sampled.t[sampled.adc], native, rtol=1e-14, atol=0)
    assert np.allclose(native, 1e-4 + np.linspace(0, 1e-3, 5), rtol=1e-15, atol=0)


def test_generalized_encoding_sizes(oracle):
    hoseq = HO_Sequence(W.compatibility_events())
    seqd, rf_start, rf_sign, adc_times = homs._kspace_inputs(hoseq, 1.0, None, None, GAMMA)
    k, kq = oracle.grad2kspace_np(seqd, rf_start, rf_sign, q_times=adc_times)
    assert k.shape == (seqd.nnodes - 1, 19) and kq.shape == (5, 19)
    assert np.all(k == 0) and np.all(kq == 0)
    assert rf_sign == [] or rf_sign == [0]  # one excitation pulse at the start


# -- the reference's known answers through the oracle (:55-136) -----------------

def _oracle_signal(oracle, obj, hoseq, mask, params=None, state=None):
    seqd = discretize(hoseq, sampling_params=params or {})
    parts, exc = get_sim_ranges(seqd)
    xy0 = None if state is None else state[0]
    z0 = None if state is None else state[1]
    sig, xy, z = oracle.simulate_c(obj, seqd, parts, exc, BlochHighOrder(mask).flags, xy0, z0)
    return sig, xy, z


def test_legacy_ninety_degree_pulse_known_answer(oracle):
    hoseq = HO_Sequence(W.compatibility_events())
    obj = W.compatibility_event_phantom()
    sig, xy, _ = _oracle_signal(oracle, obj, hoseq, "0000")
    expected = 1j * (obj.rho @ obj.csm)
    assert sig.shape == (5, 2)
    assert np.allclose(sig, np.tile(expected, (5, 1)), atol=1e-12, rtol=0)
    assert np.allclose(xy, 1j * obj.rho, atol=1e-12, rtol=0)


def test_measured_zeroth_order_phase_known_answer(oracle):
    seq = W.compatibility_events()
    hoseq = HO_Sequence(seq)
    obj = W.compatibility_event_phantom()
    hoseq.GR_dfc[0, 1] = Grad(20 / GAMMA, 1e-3)
    sig, _, _ = _oracle_signal(oracle, obj, hoseq, "1000")
    expected = 1j * (obj.rho @ obj.csm)
    readout = get_adc_sampling_times(seq) - seq.DUR[0]
    want = np.exp(-2j * np.pi * 20 * readout)[:, None] * expected[None, :]
    assert np.allclose(sig, want, atol=1e-12, rtol=0)
    # a measured field during the RF block must not change the excitation
    hoseq.GR_dfc[0, 0] = Grad(30 / GAMMA, seq.DUR[0])
    unchanged, _, _ = _oracle_signal(oracle, obj, hoseq, "1000")
    assert np.allclose(unchanged, sig, atol=1e-12, rtol=0)


def test_rf_acquisition_events_count_every_sample():
    for n1, n2, npre in ((3, 2, 11), (1, 0, 0), (0, 4, 5), (2, 2, 0)):
        seq = W.rf_acquisition_events(n1, n2, npre)
        seqd, comp, native = homs._sampled(HO_Sequence(seq), {})
        assert native == n1 + n2 + npre and comp is None
        parts, _ = get_sim_ranges(seqd)
        assert sum(count_block_adc(seqd.adc, parts)) == native
        assert np.allclose(seqd.t[seqd.adc], get_adc_sampling_times(seq), rtol=1e-14, atol=1e-18)


# -- closed-form properties on seeded sequences -------------------------------------

@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("dt", [1e-3, 1e-4, 2.5e-5])
def test_gre_sampling_properties(seed, dt):
    hoseq = W.gre_events(seed=seed, ntr=2, nadc=32)
    rule = MaxStepSizeRule(dt, 5e-5)
    sd = discretize(hoseq, sampling_rule=rule)
    seq = hoseq.simulation_sequence()
    t, d = sd.t, sd.dt
    assert np.all(d >= 0) and np.all(np.diff(t) >= -1e-15)
    assert np.allclose(d, np.diff(t), rtol=0, atol=1e-15 * max(1.0, t[-1]))
    assert math.isclose(t[-1], float(np.sum(seq.DUR)), rel_tol=1e-13)
    # step limits: dt outside RF pulses, dt_rf inside
    assert d.max() <= dt * (1 + 1e-9)
    assert d[sd.excitation].max() <= min(dt, 5e-5) * (1 + 1e-9)
    # exact areas of every gradient and field channel (trapezoid is exact on linear pieces)
    for i, row in enumerate((sd.gx, sd.gy, sd.gz)):
        want = sum(g.area() for g in seq.GR[i])
        assert abs(_trapz(d, row) - want) <= 1e-12 * max(1e-12, sum(abs(g.area()) for g in seq.GR[i]))
    for i in range(16):
        want = sum(g.area() for g in hoseq.GR_dfc[i])
        scale = sum(abs(g.area()) for g in hoseq.GR_dfc[i])
        assert abs(_trapz(d, sd.h[i]) - want) <= 1e-12 * max(scale, 1e-30)
    # ADC samples: exact times, each owned once
    native = get_adc_sampling_times(seq)
    assert np.allclose(t[sd.adc], native, rtol=1e-14, atol=0)
    parts, _ = get_sim_ranges(sd)
    assert sum(count_block_adc(sd.adc, parts)) == native.shape[0]
    # RF: excitation intervals cover exactly the pulses, B1 area close to the shape's integral
    pulses = [(j, seq.RF[0, j]) for j in range(len(seq)) if seq.RF[0, j].is_on()]
    assert math.isclose(float(d[sd.excitation].sum()), sum(float(np.sum(r.T)) for _, r in pulses), rel_tol=1e-12)
    area = complex(np.sum(sd.b1[:-1][sd.excitation] * d[sd.excitation]))
    want = sum(complex(np.sum((r.knots()[1][1:] + r.knots()[1][:-1]) * np.diff(r.knots()[0])) / 2) for _, r in pulses)
    assert abs(area - want) <= 2e-2 * abs(want)
    assert np.all(sd.df[:-1][sd.excitation] != 0)


def test_hard_pulse_area_is_exact():
    tau = 3.3e-4
    seq = Sequence([[Grad(0.0, 0.0)]] * 3, [RF(0.7e-6 * np.exp(0.3j), tau, 0.0, 2e-5)], [ADC(4, 1e-4, 2e-4)])
    sd = discretize(HO_Sequence(seq))
    area = complex(np.sum(sd.b1[:-1][sd.excitation] * sd.dt[sd.excitation]))
    assert abs(area - 0.7e-6 * np.exp(0.3j) * tau) <= 1e-15 * 0.7e-6 * tau
    assert math.isclose(rf_pulses(seq)[0][1], 360 * GAMMA * 0.7e-6 * tau, rel_tol=1e-13)
    assert math.isclose(rf_pulses(seq)[0][0], 2e-5 + tau / 2, rel_tol=1e-15)


def test_boundary_merge_rule():
    # continuous boundary (ramps to zero): the blocks share one node
    a = Sequence([[Grad(1e-3, 1e-3, 1e-4)], [Grad(0.0, 0.0)], [Grad(0.0, 0.0)]])
    s1 = discretize(HO_Sequence(a))
    s2 = discretize(HO_Sequence(a + a))
    assert s2.nnodes == 2 * s1.nnodes - 1
    assert np.all(s2.dt > 0)
    # a jump at the boundary keeps both sides at one time
    b = Sequence([[Grad(1e-3, 1e-3)], [Grad(0.0, 0.0)], [Grad(0.0, 0.0)]])
    s3 = discretize(HO_Sequence(b + b))
    zero = np.flatnonzero(s3.dt == 0)
    assert zero.shape[0] >= 1
    assert math.isclose(_trapz(s3.dt, s3.gx), 2e-6, rel_tol=1e-13)


def test_adc_on_the_first_node_is_kept():
    seq = Sequence([[Grad(0.0, 0.0)]] * 3, None, [ADC(3, 1e-3)])
    seqd, _, native = homs._sampled(HO_Sequence(seq), {})
    parts, _ = get_sim_ranges(seqd)
    assert native == 3 and sum(count_block_adc(seqd.adc, parts)) == 3
    assert seqd.t[0] == 0 and seqd.dt[0] == 0 and not seqd.adc[0]


def test_colliding_adc_samples_are_a_count_mismatch():
    seq = Sequence([[Grad(0.0, 0.0)]] * 3, None, [ADC(2, 0.0, 1e-4)], [1e-3])
    obj = W.compatibility_event_phantom()
    seqd, _, native = homs._sampled(HO_Sequence(seq), {})
    with pytest.raises(DimensionMismatch, match="ADC count"):
        homs._setup(obj, seqd, {}, None, None, native)


# -- constructors, arithmetic, errors -----------------------------------------------

def test_constructor_forms_and_durations():
    assert len(HO_Sequence()) == 1
    seq = W.compatibility_events()
    h = HO_Sequence(seq)
    assert h.GR_dfc.shape == (16, 2) and np.allclose(h.DUR, [1e-4, 2e-3])
    h2 = HO_Sequence(seq[0], [Grad(1.0, 5e-4)], 3e-4)
    assert h2.GR_dfc.shape == (16, 1) and math.isclose(h2.DUR[0], 5e-4)
    h3 = HO_Sequence(seq[1], [Grad(1.0, 1e-3)], 5e-3)
    assert math.isclose(h3.DUR[0], 5e-3)
    with pytest.raises(ArgumentError):
        HO_Sequence([[Grad(0.0, 1e-3)]] * 17)
    with pytest.raises(DimensionMismatch):
        HO_Sequence(seq, [[Grad(0.0, 1e-3)]])
    with pytest.raises(ArgumentError):
        Grad(1.0, -1e-3)
    with pytest.raises(ArgumentError):
        ADC(-1, 1e-3)
    with pytest.raises(DimensionMismatch):
        Grad([1.0, 2.0, 3.0], [1e-3])
    with pytest.raises(ArgumentError):
        discretize(h, freq_in_phase=True)
    with pytest.raises(ArgumentError):
        MaxStepSizeRule(0.0, 1e-5)


def test_arithmetic_and_indexing():
    h = W.gre_events(seed=5, ntr=1, nadc=8)
    n = len(h)
    assert len(h + h) == 2 * n
    assert len(h[0]) == 1 and len(h[0:3]) == 3
    assert h[np.zeros(n, bool)] is None
    neg = -h
    assert neg.GR_dfc[1, 0].area() == -h.GR_dfc[1, 0].area()
    assert neg.SEQ.GR[2, 0].area() == -h.SEQ.GR[2, 0].area()
    two = 2.0 * h
    assert math.isclose(two.SEQ.GR[2, 0].area(), 2 * h.SEQ.GR[2, 0].area())
    c = h * 1j
    assert np.allclose(c.SEQ.RF[0, 0].A, 1j * np.asarray(h.SEQ.RF[0, 0].A))
    assert c.GR_dfc[1, 0] is h.GR_dfc[1, 0]
    half = h / 2
    assert math.isclose(half.GR_dfc[1, 0].area(), h.GR_dfc[1, 0].area() / 2)
    assert len(list(iter(h))) == n
    assert np.allclose(get_block_start_times(h.SEQ)[-1], np.sum(h.SEQ.DUR))


def test_adc_phase_compensation():
    seq = Sequence([[Grad(0.0, 0.0), Grad(0.0, 0.0)]] * 3, None, [ADC(2, 1e-3, 0.0, 0.0, 0.4), ADC(3, 1e-3)])
    comp = get_adc_phase_compensation(seq)
    assert comp.dtype == np.complex64 and comp.shape == (5,)
    assert np.allclose(comp[:2], np.exp(-0.4j), rtol=1e-7) and np.all(comp[2:] == 1)
    seqd, c, native = homs._sampled(HO_Sequence(seq), {})
    assert native == 5 and c is not None


def test_preserved_samples_follow_the_rule():
    n = 201
    shape = np.sinc(np.linspace(-3, 3, n)).astype(np.complex128) * 1e-6
    wave = 1e-3 * np.sin(np.linspace(0, 6, 97))
    seq = Sequence([[Grad(wave, 2e-3, 0.0, 0.0, 1.3e-3)], [Grad(0.0, 0.0)], [Grad(0.0, 0.0)]],
                   [RF(shape, 1e-3, 0.0, 2e-4)],
                   [ADC(0, 0.0)])
    hoseq = HO_Sequence(seq)
    default = discretize(hoseq, sampling_rule=MaxStepSizeRule(1e-3, 5e-5))
    exc = int(default.excitation.sum())
    assert exc == 20  # 1 ms at 50 us, the centre falling on the grid
    assert math.isclose(default.t[np.flatnonzero(default.excitation)[0]], 2e-4, rel_tol=1e-12)
    every = discretize(hoseq, sampling_rule=MaxStepSizeRule(1e-3, 5e-5, ("gradients", "rf_center", "rf")))
    assert int(every.excitation.sum()) == n - 1
    # the nominal waveform's knots are nodes by default, so its area is exact; without them it is sampled
    area = seq.GR[0, 0].area()
    assert abs(_trapz(default.dt, default.gx) - area) <= 1e-12 * abs(area)
    coarse = discretize(hoseq, sampling_rule=MaxStepSizeRule(1e-3, 5e-5, ("rf_center",)))
    assert coarse.nnodes < default.nnodes
    knots = seq.GR[0, 0].knots()[0]
    assert not np.all(np.isin(np.round(knots[2:-2], 12), np.round(coarse.t, 12)))
    with pytest.raises(ArgumentError):
        MaxStepSizeRule(1e-3, 5e-5, ("adc",))


def test_repeated_blocks_sample_once_and_identically():
    """Blocks sharing their event objects are sampled once; the result equals
    the same sequence built from distinct, equal events."""
    import copy

    def tr(fresh):
        mk = (lambda e: copy.deepcopy(e)) if fresh else (lambda e: e)
        return (Sequence([[mk(exc_g)], [mk(zero)], [mk(ss)]], [mk(rf)], [mk(no_adc)])
                + Sequence([[mk(ro)], [mk(zero)], [mk(zero)]], None, [mk(adc)]))

    zero, no_adc = Grad(0.0, 0.0), ADC(0, 0.0)
    exc_g, ss = Grad(0.0, 0.0), Grad(5e-3, 1e-3, 1e-4)
    rf = RF(np.sinc(np.linspace(-2, 2, 41)) * 2e-6, 1e-3, 0.0, 1e-4)
    ro, adc = Grad(4e-3, 2e-3, 1e-4), ADC(64, 2e-3 - 3e-5, 1e-4)
    shared = tr(False)
    for _ in range(199):
        shared = shared + tr(False)
    distinct = tr(True)
    for _ in range(199):
        distinct = distinct + tr(True)
    a = discretize(HO_Sequence(shared))
    b = discretize(HO_Sequence(distinct))
    for k in ("t", "dt", "gx", "gy", "gz", "b1", "df", "adc", "excitation", "h"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert int(a.adc.sum()) == 200 * 64


def test_sequence_display_and_event_samples():
    """HO_Sequence's summary (HO_Sequence.jl:139-147) and get_samples (:169-200)."""
    from homs.sequence import get_samples
    h = HO_Sequence(W.compatibility_events())
    assert repr(h) == "HO_Sequence[ τ = 2.1 ms | blocks: 2 | ADC: 1 | GR: 0 | RF: 1 | DEF: 0 ]"
    g = get_samples(h)
    assert set(g) == {f"h{k}" for k in range(16)} | {"gx", "gy", "gz", "rf", "adc"}
    assert np.allclose(g["adc"][0], get_adc_sampling_times(h.SEQ)) and np.all(g["adc"][1] == 1)
    t, a = g["rf"]
    assert t[1] == 0 and np.isclose(a[1].real, 1 / (4 * GAMMA * 1e-4))
    h.GR_dfc[0, 1] = Grad(2e-7, 1e-3)
    t0, a0 = get_samples(h)["h0"]
    assert np.isclose(t0.max(), 1.1e-3) and np.isclose(a0.max(), 2e-7)
    assert np.all(get_samples(h, off_val=np.inf)["h3"][1] == np.inf)


def test_rf_sampling_converges(oracle):
    """Halving dt_rf roughly halves the change of the signal: a shaped pulse is
    sampled at dt_rf with the engine's left-point excitation rule (first order)."""
    hoseq = W.gre_events(seed=4, ntr=1, nadc=32)
    obj, _, _ = W.high_order_workload(nspins=64, nsteps=4, ncoils=2)
    sig = []
    for dt_rf in (1e-4, 5e-5, 2.5e-5, 1.25e-5):
        sd = discretize(hoseq, sampling_rule=MaxStepSizeRule(1e-4, dt_rf))
        parts, exc = get_sim_ranges(sd)
        sig.append(oracle.simulate_c(obj, sd, parts, exc, BlochHighOrder("1111").flags)[0])
    d = [np.linalg.norm(sig[i + 1] - sig[i]) for i in range(3)]
    assert d[1] < 0.7 * d[0] and d[2] < 0.7 * d[1]


def test_native_sequence_is_accepted_as_high_order_sequence():
    import homs
    seq = W.compatibility_events()
    a, comp_a, na = homs._sampled(seq, {})
    b, comp_b, nb = homs._sampled(HO_Sequence(seq), {})
    assert na == nb == 5 and comp_a is None and comp_b is None
    for k in ("t", "dt", "gx", "b1", "adc", "excitation", "h"):
        assert np.array_equal(getattr(a, k), getattr(b, k))
    with pytest.raises(ArgumentError, match="Sequence"):
        homs._sampled("not a sequence", {})
