"""Randomised properties of ``discretize`` (CPU, hypothesis): on sequences of
random trapezoids (zero and non-zero ramps, delays), sampled waveforms, hard and
shaped pulses with delays, ADC windows inside and outside the pulses, measured
fields and zero-length blocks, the sampled sequence keeps its invariants:
non-negative intervals with consistent lengths, the exact area of every
gradient and field channel, the exact ADC times each owned once, the RF support
covered exactly by excitation intervals, and the step limits."""
import math
import os

import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import HealthCheck, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402

from homs.model import count_block_adc, get_sim_ranges  # noqa: E402
from homs.sequence import (ADC, RF, Grad, HO_Sequence, MaxStepSizeRule, Sequence, discretize,  # noqa: E402
                           get_adc_sampling_times)

US = 1e-6
times = st.integers(min_value=0, max_value=400).map(lambda n: n * 5 * US)  # 5 us raster
amps = st.floats(min_value=-5e-3, max_value=5e-3, allow_nan=False)


@st.composite
def grads(draw):
    kind = draw(st.sampled_from(["zero", "trap", "wave"]))
    if kind == "zero":
        return Grad(0.0, 0.0)
    delay, rise, fall = draw(times), draw(st.sampled_from([0.0, 10 * US, 50 * US])), \
        draw(st.sampled_from([0.0, 20 * US]))
    if kind == "trap":
        return Grad(draw(amps), draw(times), rise, fall, delay)
    n = draw(st.integers(min_value=2, max_value=9))
    return Grad(np.array([draw(amps) for _ in range(n)]), draw(times) + 10 * US, rise, fall, delay)


@st.composite
def blocks(draw):
    gr = [draw(grads()) for _ in range(3)]
    if draw(st.booleans()):
        t_rf = draw(times) + 20 * US
        if draw(st.booleans()):
            rf = RF(complex(draw(st.floats(1e-7, 5e-6)), draw(st.floats(-1e-6, 1e-6))), t_rf, 0.0, draw(times))
        else:
            n = draw(st.integers(min_value=3, max_value=21))
            rf = RF(np.hanning(n + 2)[1:-1] * draw(st.floats(1e-7, 5e-6)), t_rf, draw(st.floats(-50, 50)),
                    draw(times))
    else:
        rf = RF(0.0, 0.0)
    if draw(st.booleans()):
        adc = ADC(draw(st.integers(min_value=1, max_value=12)), draw(times) + 5 * US, draw(times))
    else:
        adc = ADC(0, 0.0)
    dur = draw(st.sampled_from([None, 0.0]))
    return gr, rf, adc, dur


@st.composite
def sequences(draw):
    nb = draw(st.integers(min_value=1, max_value=6))
    bl = [draw(blocks()) for _ in range(nb)]
    gr = [[b[0][i] for b in bl] for i in range(3)]
    rf = [b[1] for b in bl]
    adc = [b[2] for b in bl]
    ev = [max([g.dur for g in b[0]] + [b[1].dur, b[2].dur]) for b in bl]
    dur = [e if b[3] is None else e + b[3] for b, e in zip(bl, ev)]
    seq = Sequence(gr, rf, adc, dur)
    fields = [[draw(grads()) if (k < 4 and draw(st.booleans())) else Grad(0.0, 0.0) for _ in range(nb)]
              for k in range(16)]
    return HO_Sequence(seq, fields)


def _trapz(dt, x):
    return float(np.sum((x[1:] + x[:-1]) / 2 * dt))


@settings(max_examples=int(os.environ.get("HOMS_HYPOTHESIS_EXAMPLES", "60")), deadline=None,
          suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large])
@given(sequences(), st.sampled_from([1e-4, 2.5e-5]))
def test_discretize_invariants(hoseq, dt):
    seq = hoseq.simulation_sequence()
    adc_times = get_adc_sampling_times(seq)
    if np.unique(np.round(adc_times, 13)).shape[0] != adc_times.shape[0]:
        return  # two ADC samples at one time: a count mismatch the engine reports, not a sampling case
    sd = discretize(hoseq, sampling_rule=MaxStepSizeRule(dt, 5e-5))
    n = sd.nnodes
    assert sd.dt.shape == (n - 1,) and sd.excitation.shape == (n - 1,) and sd.h.shape == (16, n)
    assert np.all(sd.dt >= 0)
    assert math.isclose(float(sd.t[-1]), float(np.sum(seq.DUR)), rel_tol=1e-12, abs_tol=1e-15)
    if n > 1:
        assert sd.dt.max() <= dt * (1 + 1e-9) + 1e-15
        if sd.excitation.any():
            assert sd.dt[sd.excitation].max() <= min(dt, 5e-5) * (1 + 1e-9) + 1e-15
    for i, row in enumerate((sd.gx, sd.gy, sd.gz)):
        want = sum(g.area() for g in seq.GR[i])
        scale = sum(abs(g.area()) for g in seq.GR[i]) + 1e-30
        assert abs(_trapz(sd.dt, row) - want) <= 1e-11 * scale
    for k in range(16):
        want = sum(g.area() for g in hoseq.GR_dfc[k])
        scale = sum(abs(g.area()) for g in hoseq.GR_dfc[k]) + 1e-30
        assert abs(_trapz(sd.dt, sd.h[k]) - want) <= 1e-11 * scale
    assert np.allclose(sd.t[sd.adc], adc_times, rtol=0, atol=1e-15)
    if n > 1:
        parts, _ = get_sim_ranges(sd)
        assert sum(count_block_adc(sd.adc, parts)) == adc_times.shape[0]
    on = [r for r in seq.RF.ravel() if r.is_on()]
    assert math.isclose(float(sd.dt[sd.excitation].sum()), sum(float(np.sum(r.T)) for r in on), rel_tol=1e-12,
                        abs_tol=1e-15)
