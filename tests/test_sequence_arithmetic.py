"""HO_Sequence arithmetic, after the reference's test/unit/test_sequence_arithmetic.jl:
complex scaling moves only the RF, subtraction is concatenation with a negated
second operand, division scales every field channel, the operands stay as they
were, and the sampled sequences and (through the oracle) the signals agree."""
import copy

import numpy as np
import pytest

from homs import workloads as W
from homs.model import BlochHighOrder, get_sim_ranges
from homs.sequence import Grad, HO_Sequence, Sequence, discretize

EPS = np.finfo(np.float64).eps


def _pair():
    native = W.compatibility_events()
    gradients = [[Grad(0.0, 0.0) if block == 0 else Grad(axis * 1e-3, 1e-3) for block in range(2)]
                 for axis in range(1, 4)]
    seq = Sequence(gradients, native.RF, native.ADC, native.DUR)
    fields = [[Grad(term * 1e-6, float(seq.DUR[0])) if block == 0 else
               Grad(np.array([0, 1, -0.25, 0]) * term * 1e-5, 1e-3) for block in range(2)] for term in range(1, 17)]
    x = HO_Sequence(seq, fields)
    return x, 1.5 * x


def _grads_close(a, b):
    ta, aa = a.knots()
    tb, ab = b.knots()
    return np.allclose(ta, tb, rtol=0, atol=0) and np.allclose(aa, ab, rtol=10 * EPS, atol=0)


def _seq_close(a, b):
    return (a.GR.shape == b.GR.shape and all(_grads_close(g, h) for g, h in zip(a.GR.ravel(), b.GR.ravel()))
            and all(np.allclose(np.asarray(r.A), np.asarray(s.A), rtol=10 * EPS) for r, s in
                    zip(a.RF.ravel(), b.RF.ravel())) and np.array_equal(a.DUR, b.DUR))


def _event_samples_equal(a, b, rtol=10 * EPS):
    from homs.sequence import get_samples
    sa, sb = get_samples(a), get_samples(b)
    for name in sb:
        assert np.array_equal(sa[name][0], sb[name][0]), name
        assert np.allclose(sa[name][1], sb[name][1], rtol=rtol, atol=0), name


def _sampled_equal(a, b, rtol=10 * EPS):
    sa, sb = discretize(a), discretize(b)
    assert np.array_equal(sa.t, sb.t) and np.array_equal(sa.adc, sb.adc)
    assert np.array_equal(sa.excitation, sb.excitation)
    for k in ("gx", "gy", "gz", "h", "b1"):
        assert np.allclose(getattr(sa, k), getattr(sb, k), rtol=rtol, atol=0), k


def test_complex_rf_scaling_and_empty_iteration():
    x, _ = _pair()
    alpha = complex(0.5, -0.25)
    for scaled in (alpha * x, x * alpha):
        assert _seq_close(scaled.SEQ, x.SEQ * alpha)
        assert all(_grads_close(g, h) for g, h in zip(scaled.GR_dfc.ravel(), x.GR_dfc.ravel()))
        assert np.array_equal(scaled.DUR, x.DUR)
    empty = HO_Sequence(x.SEQ[slice(0, 0)])
    assert len(empty) == 0 and list(iter(empty)) == [] and empty.size == (0,)


def test_subtraction_is_concatenation_with_negation():
    x, y = _pair()
    ox, oy = copy.deepcopy(x), copy.deepcopy(y)
    actual, expected = x - y, x + (-y)
    assert _seq_close(actual.SEQ, x.SEQ - y.SEQ) and _seq_close(actual.SEQ, expected.SEQ)
    assert np.array_equal(actual.DUR, np.concatenate([x.DUR, y.DUR])) and np.array_equal(actual.DUR, expected.DUR)
    assert all(_grads_close(g, h) for g, h in zip(actual.GR_dfc.ravel(), expected.GR_dfc.ravel()))
    assert [r.A for r in actual.SEQ.RF.ravel()] == [r.A for r in np.concatenate([x.SEQ.RF, y.SEQ.RF], 1).ravel()]
    assert [a.N for a in actual.SEQ.ADC] == [a.N for a in np.concatenate([x.SEQ.ADC, y.SEQ.ADC])]
    _sampled_equal(actual, expected)
    _event_samples_equal(actual, expected)
    assert _seq_close(x.SEQ, ox.SEQ) and _seq_close(y.SEQ, oy.SEQ)
    assert np.array_equal(x.DUR, ox.DUR) and np.array_equal(y.DUR, oy.DUR)


@pytest.mark.parametrize("alpha", [2.0, -3.0])
def test_division_scales_every_field_channel(alpha):
    x, _ = _pair()
    actual, expected = x / alpha, (1 / alpha) * x
    assert _seq_close(actual.SEQ, x.SEQ / alpha) and _seq_close(actual.SEQ, expected.SEQ)
    assert np.array_equal(actual.DUR, x.DUR)
    for g, e, o in zip(actual.GR_dfc.ravel(), expected.GR_dfc.ravel(), x.GR_dfc.ravel()):
        assert _grads_close(g, e)
        assert np.allclose(np.asarray(g.A), np.asarray(o.A) / alpha, rtol=10 * EPS, atol=0)
    _sampled_equal(actual, expected)
    _event_samples_equal(actual, expected)


@pytest.mark.parametrize("orders", ["0000", "1111"])
def test_signal_parity_through_the_oracle(oracle, orders):
    x, y = _pair()
    obj = W.compatibility_event_phantom()
    for actual, expected in ((x - y, x + (-y)), (x / 2.0, 0.5 * x)):
        sig = []
        for s in (actual, expected):
            sd = discretize(s)
            parts, exc = get_sim_ranges(sd)
            sig.append(oracle.simulate_c(obj, sd, parts, exc, BlochHighOrder(orders).flags)[0])
        assert np.allclose(sig[0], sig[1], rtol=10 * EPS, atol=10 * EPS)
