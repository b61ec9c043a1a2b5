"""Event-level sequences and their discretisation onto one time grid.

``HO_Sequence`` mirrors src/datatypes/HO_Sequence.jl:44-120 (a KomaMRI
``Sequence`` plus a 16 x Nblocks matrix of measured field waveforms and one
duration per block) and ``discretize`` mirrors the high-order sampler of
src/datatypes/HO_DiscreteSequence.jl:82-179.  The event types they build on
(``Grad``, ``RF``, ``ADC``, ``Sequence``) belong to KomaMRIBase 0.15.2, which
the reference does not vendor; their published definitions are restated here:

* ``Grad(A, T, rise=0, fall=rise, delay=0, first=0, last=0)``: a trapezoid
  (scalar ``A``) or a uniformly sampled waveform (vector ``A`` over ``T``, or
  over the segment durations of a vector ``T`` of length len(A) - 1), with
  linear ramps from ``first`` and to ``last``.  Knots
  ``delay + [0, rise, rise + T, rise + T + fall]``, amplitudes
  ``[first, A, A, last]``; a zero rise or fall is a jump (two knots at one
  time).  Duration ``delay + rise + sum(T) + fall``.
* ``RF(A, T, df=0, delay=0, center=None)``: complex B1 (T); a hard pulse
  (scalar ``A``) or a piecewise-linear shape (vector ``A`` over ``T``), zero
  outside ``[delay, delay + T]``, frequency offset ``df`` (Hz) on its
  support.  Its centre is ``delay + T/2`` for a hard pulse, else ``delay +
  center`` or the midpoint of the first and last samples within 1e-5 of the
  largest magnitude (the peak plateau).  Flip angle
  ``360 gamma |integral B1 dt|`` degrees; up to 90.01 degrees it is an
  excitation, above a refocusing pulse.
* ``ADC(N, T, delay=0, df=0, phi=0)``: samples at ``delay + T/2`` (N = 1) or
  ``delay + linspace(0, T, N)``; the signal of an ADC with phase ``phi`` is
  multiplied by ``exp(-i phi)`` (single-precision factors) after the
  simulation.
* ``Sequence(GR, RF, ADC, DUR)``: 3 x N gradients, 1 x N pulses, N ADCs and
  N block durations (default: the longest event of each block).

KomaMRIBase's sampling internals are not vendored either, so the node
placement below is this module's own rule.  It keeps every behaviour the
reference's sampling tests fix (test/unit/test_koma_compatibility.jl:11-53):
the waveforms' own sample times are nodes even without nominal gradients,
field jumps keep both sides at one time (a zero interval), every ADC sample
is a node at its exact time, one node per time point for every field, one
``dt`` and ``excitation`` value per interval, and the boundary merge of
HO_DiscreteSequence.jl:98-131.  Per block, in block time:

1. Breakpoints: 0, the block duration, every knot of the 16 measured field
   waveforms, the RF pulse's start and end and every ADC sample time; by
   default (``MaxStepSizeRule.preserve_samples``, as the reference's
   ``(:gradients, :rf_center)``) also every knot of the 3 nominal gradients
   and the RF centre, and on request every sample of a shaped pulse.  Times
   closer than 1e-12 s are one time.
2. Between consecutive breakpoints, uniform nodes at most ``min(dt, dt_rf)``
   apart inside the RF pulse and ``dt`` apart elsewhere (``MaxStepSizeRule``,
   defaults 1e-3 s and 5e-5 s as in HO_DiscreteSequence.jl:82-89).
3. Where a gradient or field waveform jumps, two nodes at one time carry its
   left and right limits (the interval between them has dt = 0); elsewhere a
   node carries the right limit.  Waveforms are linear between knots, so the
   trapezoidal integral over the nodes equals each waveform's exact area.
4. Interval n takes B1 and df from node n (the engine's excitation rule); an
   interval is an excitation interval when it has dt > 0 and lies inside the
   RF pulse.  ADC flags sit on the last node at each ADC time.

Blocks join as in HO_DiscreteSequence.jl:98-131: a block's first node merges
into the previous block's last node when both have one time and equal samples
(every field, B1, df, ADC flag); otherwise a zero interval without excitation
joins them.  If the first node of the sequence carries an ADC sample, a copy
without it is put in front, so that the block plan (which counts ADC samples
from each block's second node on) keeps the sample.
"""
from __future__ import annotations

import math
from typing import List, Optional

import numpy as np

from .model import GAMMA, ArgumentError, DimensionMismatch, HO_DiscreteSequence

__all__ = [
    "Grad", "RF", "ADC", "Sequence", "HO_Sequence", "MaxStepSizeRule", "discretize", "get_block_start_times",
    "get_adc_sampling_times", "get_adc_phase_compensation", "rf_pulses", "validate_high_order_sequence", "get_samples",
]

_TOL = 1e-12  # seconds: sample times closer than this are one time


def _real(x, name):
    try:
        v = float(x)
    except (TypeError, ValueError):
        raise ArgumentError(f"{name} must be a real number.") from None
    if not math.isfinite(v):
        raise ArgumentError(f"{name} must be finite.")
    return v


def _nonneg(x, name):
    v = _real(x, name)
    if v < 0:
        raise ArgumentError(f"{name} must be nonnegative.")
    return v


def _durations(T, n, name):
    """Segment durations of a sampled waveform with n samples."""
    if np.ndim(T) == 0:
        T = _nonneg(T, name)
        return np.full(n - 1, T / (n - 1)) if n > 1 else np.zeros(0)
    T = np.asarray(T, dtype=np.float64).reshape(-1)
    if T.shape[0] != n - 1:
        raise DimensionMismatch(f"A sampled waveform with {n} samples needs {n - 1} segment durations.")
    if not np.all(np.isfinite(T)) or np.any(T < 0):
        raise ArgumentError(f"{name} must be finite and nonnegative.")
    return T


class Grad:
    """Gradient (or field-coefficient) waveform of one block (KomaMRIBase ``Grad``)."""

    __slots__ = ("A", "T", "rise", "fall", "delay", "first", "last")

    def __init__(self, A, T, rise=0.0, fall=None, delay=0.0, first=0.0, last=0.0):
        if np.ndim(A) == 0:
            self.A = _real(A, "A")
            if np.ndim(T) != 0:
                raise ArgumentError("A scalar gradient amplitude needs a scalar duration.")
            self.T = _nonneg(T, "T")
        else:
            a = np.asarray(A, dtype=np.float64).reshape(-1)
            if a.shape[0] == 0 or not np.all(np.isfinite(a)):
                raise ArgumentError("A sampled gradient needs finite samples.")
            self.A = a
            if a.shape[0] == 1:
                self.T = _nonneg(T, "T")
            else:
                _durations(T, a.shape[0], "T")
                self.T = _nonneg(T, "T") if np.ndim(T) == 0 else np.asarray(T, dtype=np.float64).reshape(-1).copy()
        self.rise = _nonneg(rise, "rise")
        self.fall = self.rise if fall is None else _nonneg(fall, "fall")
        self.delay = _nonneg(delay, "delay")
        self.first = _real(first, "first")
        self.last = _real(last, "last")

    @classmethod
    def zero(cls) -> "Grad":
        """A fresh ``Grad(0.0, 0.0)`` (built without argument checks)."""
        g = cls.__new__(cls)
        g.A, g.T, g.rise, g.fall, g.delay, g.first, g.last = 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0
        return g

    def _copy(self, scale: float) -> "Grad":
        g = Grad.__new__(Grad)
        g.A = self.A * scale if np.ndim(self.A) == 0 else np.asarray(self.A) * scale
        g.T = self.T if np.ndim(self.T) == 0 else np.asarray(self.T).copy()
        g.rise, g.fall, g.delay = self.rise, self.fall, self.delay
        g.first, g.last = self.first * scale, self.last * scale
        return g

    def __mul__(self, a):
        if isinstance(a, (complex, np.complexfloating)):
            return NotImplemented
        return self._copy(_real(a, "scale"))

    __rmul__ = __mul__

    def __neg__(self):
        return self._copy(-1.0)

    def __truediv__(self, a):
        return self._copy(1.0 / _real(a, "divisor"))

    @property
    def dur(self) -> float:
        return self.delay + self.rise + float(np.sum(self.T)) + self.fall

    def knots(self):
        """Block-time knots and amplitudes of the piecewise-linear waveform."""
        if np.ndim(self.A) == 0 or np.asarray(self.A).shape[0] == 1:
            a = float(np.asarray(self.A).reshape(-1)[0])
            T = float(np.sum(self.T))
            t = self.delay + np.array([0.0, self.rise, self.rise + T, self.rise + T + self.fall])
            return t, np.array([self.first, a, a, self.last])
        a = np.asarray(self.A)
        segs = _durations(self.T, a.shape[0], "T")
        inner = self.rise + np.concatenate([[0.0], np.cumsum(segs)])
        t = self.delay + np.concatenate([[0.0], inner, [inner[-1] + self.fall]])
        return t, np.concatenate([[self.first], a, [self.last]])

    def area(self) -> float:
        """Exact integral of the waveform (T s)."""
        t, a = self.knots()
        return float(np.sum((a[1:] + a[:-1]) * np.diff(t)) / 2)

    def is_on(self) -> bool:
        return bool(np.any(np.asarray(self.A) != 0) or self.first != 0 or self.last != 0)

    def __repr__(self):
        return (f"Grad(A={self.A!r}, T={self.T!r}, rise={self.rise}, fall={self.fall}, delay={self.delay}"
                + (f", first={self.first}, last={self.last}" if self.first or self.last else "") + ")")


class RF:
    """RF pulse of one block (KomaMRIBase ``RF``): complex B1 amplitude (T)."""

    __slots__ = ("A", "T", "df", "delay", "center")

    def __init__(self, A, T, df=0.0, delay=0.0, center=None):
        if np.ndim(A) == 0:
            a = complex(A)
            if not (math.isfinite(a.real) and math.isfinite(a.imag)):
                raise ArgumentError("RF amplitude must be finite.")
            if np.ndim(T) != 0:
                raise ArgumentError("A hard pulse needs a scalar duration.")
            self.A = a
            self.T = _nonneg(T, "T")
        else:
            a = np.asarray(A, dtype=np.complex128).reshape(-1)
            if a.shape[0] == 0 or not np.all(np.isfinite(a)):
                raise ArgumentError("A shaped RF pulse needs finite samples.")
            self.A = a
            if a.shape[0] == 1:
                self.T = _nonneg(T, "T")
            else:
                _durations(T, a.shape[0], "T")
                self.T = _nonneg(T, "T") if np.ndim(T) == 0 else np.asarray(T, dtype=np.float64).reshape(-1).copy()
        self.df = _real(df, "df")
        self.delay = _nonneg(delay, "delay")
        self.center = None if center is None else _nonneg(center, "center")

    def _copy(self, scale: complex) -> "RF":
        r = RF.__new__(RF)
        r.A = self.A * scale if np.ndim(self.A) == 0 else np.asarray(self.A) * scale
        r.T = self.T if np.ndim(self.T) == 0 else np.asarray(self.T).copy()
        r.df, r.delay, r.center = self.df, self.delay, self.center
        return r

    def __mul__(self, a):
        return self._copy(complex(a))

    __rmul__ = __mul__

    def __neg__(self):
        return self._copy(-1.0)

    def __truediv__(self, a):
        return self._copy(1.0 / complex(a))

    @property
    def dur(self) -> float:
        return self.delay + float(np.sum(self.T))

    def is_on(self) -> bool:
        return float(np.sum(self.T)) > 0 and bool(np.any(np.abs(np.asarray(self.A)) > 0))

    def knots(self):
        """Block-time knots and complex amplitudes (zero outside the pulse)."""
        if np.ndim(self.A) == 0 or np.asarray(self.A).shape[0] == 1:
            a = complex(np.asarray(self.A).reshape(-1)[0])
            T = float(np.sum(self.T))
            return self.delay + np.array([0.0, 0.0, T, T]), np.array([0, a, a, 0], dtype=np.complex128)
        a = np.asarray(self.A)
        inner = np.concatenate([[0.0], np.cumsum(_durations(self.T, a.shape[0], "T"))])
        t = self.delay + np.concatenate([[0.0], inner, [inner[-1]]])
        return t, np.concatenate([[0], a, [0]]).astype(np.complex128)

    def center_time(self) -> float:
        """Block time of the pulse centre."""
        if np.ndim(self.A) == 0 or np.asarray(self.A).shape[0] == 1:
            return self.delay + float(np.sum(self.T)) / 2
        if self.center is not None:
            return self.delay + self.center
        t, a = self.knots()
        mag = np.abs(a[1:-1])
        peak = np.flatnonzero(mag >= mag.max() * (1 - 1e-5))
        return float((t[1 + peak[0]] + t[1 + peak[-1]]) / 2)

    def flip_angle(self, gamma: float = GAMMA) -> float:
        """360 gamma |integral B1 dt| in degrees."""
        t, a = self.knots()
        return 360.0 * gamma * abs(complex(np.sum((a[1:] + a[:-1]) * np.diff(t)) / 2))

    def __repr__(self):
        return f"RF(A={self.A!r}, T={self.T!r}, df={self.df}, delay={self.delay})"


class ADC:
    """Acquisition window of one block (KomaMRIBase ``ADC``)."""

    __slots__ = ("N", "T", "delay", "df", "phi")

    def __init__(self, N, T, delay=0.0, df=0.0, phi=0.0):
        if not isinstance(N, (int, np.integer)) or isinstance(N, bool) or N < 0:
            raise ArgumentError("ADC N must be a nonnegative integer.")
        self.N = int(N)
        self.T = _nonneg(T, "T")
        self.delay = _nonneg(delay, "delay")
        self.df = _real(df, "df")
        self.phi = _real(phi, "phi")

    @property
    def dur(self) -> float:
        return self.delay + self.T

    def times(self) -> np.ndarray:
        if self.N == 0:
            return np.zeros(0)
        if self.N == 1:
            return np.array([self.delay + self.T / 2])
        return self.delay + np.linspace(0.0, self.T, self.N)

    def __repr__(self):
        return f"ADC(N={self.N}, T={self.T}, delay={self.delay})"


def _objects(x, cls, name) -> np.ndarray:
    """A numpy object array of ``cls`` instances (shape kept)."""
    if isinstance(x, cls):
        x = [x]
    arr = np.empty(np.shape(x) if not isinstance(x, np.ndarray) else x.shape, dtype=object)
    if arr.ndim == 0:
        raise ArgumentError(f"{name} must be an array of {cls.__name__} events.")
    flat_in = list(np.asarray(x, dtype=object).reshape(-1)) if isinstance(x, np.ndarray) else list(_flatten(x))
    for i, v in enumerate(flat_in):
        if not isinstance(v, cls):
            raise ArgumentError(f"{name} must contain only {cls.__name__} events.")
        arr.reshape(-1)[i] = v
    return arr


def _flatten(x):
    for v in x:
        if isinstance(v, (list, tuple)):
            yield from _flatten(v)
        else:
            yield v


class Sequence:
    """KomaMRIBase ``Sequence``: ``GR`` (3 x N Grad), ``RF`` (1 x N),
    ``ADC`` (N) and ``DUR`` (N block durations, s), plus ``DEF`` (the
    definitions of a sequence file) and ``EXT`` (one extension id per block,
    not interpreted)."""

    def __init__(self, GR=None, RF_=None, ADC_=None, DUR=None):
        if GR is None and RF_ is None and ADC_ is None and DUR is None:
            # Sequence(): no blocks, to be built up with ``seq += event``
            z = np.empty((3, 0), dtype=object)
            self.GR, self.RF, self.ADC, self.DUR = z, np.empty((1, 0), dtype=object), np.empty(0, dtype=object), \
                np.zeros(0)
            self.DEF, self.EXT = {}, np.zeros(0, dtype=np.int64)
            return
        if GR is None:
            n = len(ADC_) if ADC_ is not None else (np.shape(RF_)[-1] if RF_ is not None else len(DUR))
            GR = [[Grad(0.0, 0.0)] * n for _ in range(3)]
        gr = _objects(GR, Grad, "GR")
        if gr.ndim == 1:
            gr = gr.reshape(-1, 1)
        if gr.ndim != 2 or gr.shape[0] > 3:
            raise DimensionMismatch("GR must have at most 3 rows (x, y, z) and one column per block.")
        n = gr.shape[1]
        full = np.empty((3, n), dtype=object)
        for i in range(3):
            for j in range(n):
                full[i, j] = gr[i, j] if i < gr.shape[0] else Grad(0.0, 0.0)
        self.GR = full
        if RF_ is None:
            rf = np.empty((1, n), dtype=object)
            for j in range(n):
                rf[0, j] = RF(0.0, 0.0)
        else:
            rf = _objects(RF_, RF, "RF").reshape(1, -1) if np.ndim(RF_) <= 1 else _objects(RF_, RF, "RF")
        if rf.shape[1] != n:
            raise DimensionMismatch("RF must contain one pulse per block.")
        self.RF = rf
        if ADC_ is None:
            adc = np.empty(n, dtype=object)
            for j in range(n):
                adc[j] = ADC(0, 0.0)
        else:
            adc = _objects(ADC_, ADC, "ADC").reshape(-1)
        if adc.shape[0] != n:
            raise DimensionMismatch("ADC must contain one window per block.")
        self.ADC = adc
        if DUR is None:
            self.DUR = np.array([max([g.dur for g in self.GR[:, j]] + [r.dur for r in self.RF[:, j]]
                                     + [self.ADC[j].dur]) for j in range(n)], dtype=np.float64)
        else:
            d = np.asarray(DUR, dtype=np.float64).reshape(-1)
            if d.shape[0] != n:
                raise DimensionMismatch("DUR must contain one duration per block.")
            if not np.all(np.isfinite(d)) or np.any(d < 0):
                raise ArgumentError("Block durations must be finite and nonnegative.")
            self.DUR = d.copy()
        self.DEF = {}
        self.EXT = np.zeros(n, dtype=np.int64)

    @classmethod
    def _raw(cls, GR, RF_, ADC_, DUR, DEF=None, EXT=None) -> "Sequence":
        s = cls.__new__(cls)
        s.GR, s.RF, s.ADC, s.DUR = GR, RF_, ADC_, np.asarray(DUR, dtype=np.float64)
        s.DEF = dict(DEF or {})
        s.EXT = np.zeros(s.DUR.shape[0], dtype=np.int64) if EXT is None else np.asarray(EXT, dtype=np.int64)
        return s

    def __len__(self):
        return int(self.DUR.shape[0])

    @property
    def size(self):
        return (len(self),)

    def __getitem__(self, idx):
        if isinstance(idx, (int, np.integer)):
            idx = [int(idx)]
        return Sequence._raw(self.GR[:, idx], self.RF[:, idx], self.ADC[idx], self.DUR[idx], self.DEF, self.EXT[idx])

    @staticmethod
    def block(event) -> "Sequence":
        """One block holding a single event: an RF pulse, an ADC window or an
        x gradient (KomaMRIBase's ``seq + event``)."""
        if isinstance(event, RF):
            return Sequence([[Grad(0.0, 0.0)]] * 3, [event], [ADC(0, 0.0)])
        if isinstance(event, ADC):
            return Sequence([[Grad(0.0, 0.0)]] * 3, [RF(0.0, 0.0)], [event])
        if isinstance(event, Grad):
            return Sequence([[event], [Grad(0.0, 0.0)], [Grad(0.0, 0.0)]])
        raise ArgumentError("A block holds a Sequence, an RF, an ADC or a Grad.")

    def __add__(self, other) -> "Sequence":
        if not isinstance(other, Sequence):
            other = Sequence.block(other)
        return Sequence._raw(np.concatenate([self.GR, other.GR], axis=1), np.concatenate([self.RF, other.RF], axis=1),
                             np.concatenate([self.ADC, other.ADC]), np.concatenate([self.DUR, other.DUR]),
                             {**other.DEF, **self.DEF}, np.concatenate([self.EXT, other.EXT]))

    def _map(self, grad=None, rf=None) -> "Sequence":
        g = self.GR if grad is None else np.vectorize(grad, otypes=[object])(self.GR)
        r = self.RF if rf is None else np.vectorize(rf, otypes=[object])(self.RF)
        return Sequence._raw(g, r, self.ADC.copy(), self.DUR.copy(), self.DEF, self.EXT.copy())

    def __neg__(self):
        return self._map(grad=lambda g: -g)

    def __sub__(self, other):
        return self + (-other)

    def __mul__(self, a):
        if isinstance(a, (complex, np.complexfloating)):
            return self._map(rf=lambda r: r * a)
        return self._map(grad=lambda g: g * a)

    __rmul__ = __mul__

    def __truediv__(self, a):
        return self._map(grad=lambda g: g / a)

    def __repr__(self):
        return f"Sequence({len(self)} blocks, {float(np.sum(self.DUR)) * 1e3:.3f} ms)"


def _grad_matrix(x, vector_as_row: bool) -> np.ndarray:
    g = _objects(x, Grad, "GR_dfc")
    if g.ndim == 1:
        g = g.reshape(1, -1) if vector_as_row else g.reshape(-1, 1)
    if g.ndim != 2:
        raise DimensionMismatch("GR_dfc must be a matrix of Grad events (field channels x blocks).")
    return g


def _padded(gr: np.ndarray) -> np.ndarray:
    m, n = gr.shape
    if not 1 <= m <= 16:
        raise ArgumentError("Expected 1 to 16 high-order field channels.")
    out = np.empty((16, n), dtype=object)
    out[:m] = gr
    for i in range(m, 16):
        for j in range(n):
            out[i, j] = Grad.zero()
    return out


def _column_durations(gr: np.ndarray) -> np.ndarray:
    return np.array([max(g.dur for g in gr[:, j]) for j in range(gr.shape[1])], dtype=np.float64)


def _is_grad_array(x) -> bool:
    if isinstance(x, Grad):
        return True
    try:
        flat = list(np.asarray(x, dtype=object).reshape(-1)) if isinstance(x, np.ndarray) else list(_flatten(x))
    except TypeError:
        return False
    return len(flat) > 0 and all(isinstance(v, Grad) for v in flat)


class HO_Sequence:  # noqa: N801
    """A ``Sequence`` plus measured field waveforms (src/datatypes/HO_Sequence.jl:44-80).

    Constructors, as in the reference: ``HO_Sequence()``,
    ``HO_Sequence(GR_dfc)`` (M x N matrix, or a vector taken as one row: h0
    per block), ``HO_Sequence(SEQ)``, ``HO_Sequence(SEQ, GR_dfc)`` and
    ``HO_Sequence(SEQ, GR_dfc_vector, DUR)`` (one block).  ``GR_dfc`` has 1 to
    16 rows (h0..h15, missing rows are zero waveforms); without ``SEQ`` the
    nominal gradients are rows h1..h3.  ``DUR`` is the per-block maximum of
    the sequence's, the waveforms' and the given durations.
    """

    def __init__(self, *args):
        if len(args) == 0:
            args = ([Grad(0.0, 0.0)],)
        if len(args) == 1 and not isinstance(args[0], Sequence):
            gr = _padded(_grad_matrix(args[0], vector_as_row=True))
            seq = Sequence(gr[1:4, :])
            self._init(seq, gr, np.maximum(seq.DUR, _column_durations(gr)))
        elif len(args) == 1:
            seq = args[0]
            gr = _padded(_grad_matrix([[Grad(0.0, 0.0)] * len(seq)], vector_as_row=True))
            self._init(seq, gr, np.maximum(seq.DUR, _column_durations(gr)))
        elif len(args) == 2:
            seq, gr = args
            gr = _grad_matrix(gr, vector_as_row=False)
            self._check(seq, gr)
            gr = _padded(gr)
            self._init(seq, gr, np.maximum(seq.DUR, _column_durations(gr)))
        elif len(args) == 3:
            seq, gr, dur = args
            if np.ndim(dur) == 0:
                gr = _grad_matrix(gr, vector_as_row=False)
                dur = [dur]
            else:
                gr = _grad_matrix(gr, vector_as_row=False)
            self._check(seq, gr)
            d = np.asarray(dur, dtype=np.float64).reshape(-1)
            if d.shape[0] != len(seq):
                raise DimensionMismatch("Expected one duration per sequence block.")
            gr = _padded(gr)
            self._init(seq, gr, np.maximum(np.maximum(seq.DUR, _column_durations(gr)), d))
        else:
            raise ArgumentError("HO_Sequence takes (GR_dfc), (SEQ), (SEQ, GR_dfc) or (SEQ, GR_dfc, DUR).")

    @staticmethod
    def _check(seq, gr):
        if not isinstance(seq, Sequence):
            raise ArgumentError("SEQ must be a Sequence.")
        if len(seq) != gr.shape[1]:
            raise DimensionMismatch("The number of SEQ and GR_dfc objects must be the same.")
        if not 1 <= gr.shape[0] <= 16:
            raise ArgumentError("Expected 1 to 16 high-order field channels.")

    def _init(self, seq, gr, dur):
        self.SEQ = seq
        self.GR_dfc = gr
        self.DUR = np.asarray(dur, dtype=np.float64)

    @classmethod
    def _raw(cls, seq, gr, dur) -> "HO_Sequence":
        h = cls.__new__(cls)
        h._init(seq, gr, dur)
        return h

    def __len__(self):
        return int(self.DUR.shape[0])

    @property
    def size(self):
        return (self.GR_dfc.shape[1],)

    def __getitem__(self, idx):
        if isinstance(idx, (int, np.integer)):
            idx = [int(idx)]
        if isinstance(idx, (list, np.ndarray)) and np.asarray(idx).dtype == bool and not np.any(idx):
            return None
        return HO_Sequence._raw(self.SEQ[idx], self.GR_dfc[:, idx], self.DUR[idx])

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]

    def __add__(self, other: "HO_Sequence") -> "HO_Sequence":
        return HO_Sequence._raw(self.SEQ + other.SEQ, np.concatenate([self.GR_dfc, other.GR_dfc], axis=1),
                                np.concatenate([self.DUR, other.DUR]))

    def __neg__(self):
        return HO_Sequence._raw(-self.SEQ, np.vectorize(lambda g: -g, otypes=[object])(self.GR_dfc), self.DUR.copy())

    def __sub__(self, other):
        return self + (-other)

    def __mul__(self, a):
        if isinstance(a, (complex, np.complexfloating)):
            return HO_Sequence._raw(self.SEQ * a, self.GR_dfc.copy(), self.DUR.copy())
        return HO_Sequence._raw(self.SEQ * a, np.vectorize(lambda g: g * a, otypes=[object])(self.GR_dfc),
                                self.DUR.copy())

    __rmul__ = __mul__

    def __truediv__(self, a):
        return HO_Sequence._raw(self.SEQ / a, np.vectorize(lambda g: g / a, otypes=[object])(self.GR_dfc),
                                self.DUR.copy())

    def simulation_sequence(self) -> Sequence:
        """The native sequence with each block lasting the longest of its
        sequence, measured-field and event durations (HO_Sequence.jl:114-119).
        The caller's sequence is not modified."""
        seq = self.SEQ
        ev = np.array([max([g.dur for g in seq.GR[:, j]] + [r.dur for r in seq.RF[:, j]] + [seq.ADC[j].dur])
                       for j in range(len(seq))], dtype=np.float64)
        dur = np.maximum.reduce([seq.DUR, self.DUR, _column_durations(self.GR_dfc), ev])
        return Sequence._raw(seq.GR, seq.RF, seq.ADC, dur, seq.DEF, seq.EXT)

    def validate(self):
        validate_high_order_sequence(self)

    def __repr__(self):
        s = self.SEQ
        ngr = sum(int(g.is_on()) for g in s.GR.ravel())
        nadc = sum(int(a.N > 0) for a in s.ADC)
        nrf = sum(int(r.is_on()) for r in s.RF.ravel())
        tau = round(float(np.sum(s.DUR)) * 1e3, 3)
        return (f"HO_Sequence[ τ = {tau} ms | blocks: {len(s)} | ADC: {nadc} | GR: {ngr} | RF: {nrf} | "
                f"DEF: {len(s.DEF)} ]")


def get_samples(hoseq: HO_Sequence, off_val=0.0) -> dict:
    """Event samples of every channel in sequence time (``get_samples``,
    HO_Sequence.jl:169-200): ``"h0"``..``"h15"``, ``"gx"``, ``"gy"``, ``"gz"``
    and ``"rf"`` as (t, A) knot arrays, ``"adc"`` as (sample times, ones).
    ``off_val`` replaces zero field amplitudes (to hide them in plots)."""
    seq = hoseq.simulation_sequence()
    starts = get_block_start_times(seq)
    out = {}

    def chain(events):
        ts, vs = [], []
        for j, e in enumerate(events):
            t, a = e.knots()
            ts.append(starts[j] + t)
            vs.append(a)
        if not ts:
            return np.zeros(0), np.zeros(0)
        return np.concatenate(ts), np.concatenate(vs)

    for k in range(16):
        t, a = chain(hoseq.GR_dfc[k])
        if off_val != 0:
            a = np.where(a == 0, off_val, a)
        out[f"h{k}"] = (t, a)
    for k, name in enumerate(("gx", "gy", "gz")):
        out[name] = chain(seq.GR[k])
    out["rf"] = chain(seq.RF[0])
    t = get_adc_sampling_times(seq)
    out["adc"] = (t, np.ones_like(t))
    return out


def validate_high_order_sequence(hoseq: HO_Sequence) -> None:
    """Shape checks of HO_Sequence.jl:100-110."""
    n = len(hoseq.SEQ)
    if hoseq.GR_dfc.shape != (16, n):
        raise DimensionMismatch("Expected 16 field channels and one column per sequence block.")
    if hoseq.DUR.shape[0] != n:
        raise DimensionMismatch("Expected one duration per sequence block.")
    if hoseq.SEQ.RF.shape[0] != 1:
        raise ArgumentError("High-order sampling supports a single transmit RF channel.")


_PRESERVABLE = ("gradients", "rf_center", "rf")


class MaxStepSizeRule:
    """Largest node spacing outside (``dt``) and inside (``dt_rf``) RF
    pulses, and which event samples are kept as nodes: ``"gradients"`` (every
    knot of the nominal gradients), ``"rf_center"`` (each pulse's centre) and
    ``"rf"`` (every sample of a shaped pulse).  The default keeps gradients
    and RF centres, as the reference's rule does (HO_DiscreteSequence.jl:82-89);
    the measured field waveforms' knots, block boundaries, pulse ends and ADC
    times are always nodes."""

    def __init__(self, dt=1e-3, dt_rf=5e-5, preserve_samples=("gradients", "rf_center")):
        self.dt = _real(dt, "dt")
        self.dt_rf = _real(dt_rf, "dt_rf")
        if self.dt <= 0 or self.dt_rf <= 0:
            raise ArgumentError("Sampling steps must be positive.")
        if isinstance(preserve_samples, str):
            preserve_samples = (preserve_samples,)
        ps = tuple(str(v).lstrip(":") for v in preserve_samples)
        if not set(ps) <= set(_PRESERVABLE):
            raise ArgumentError(f"preserve_samples entries must be among {_PRESERVABLE}.")
        self.preserve_samples = ps

    def __repr__(self):
        return f"MaxStepSizeRule(dt={self.dt}, dt_rf={self.dt_rf}, preserve_samples={self.preserve_samples})"


def get_block_start_times(seq: Sequence) -> np.ndarray:
    """Block start times plus the sequence end: cumsum([0; DUR])."""
    return np.concatenate([[0.0], np.cumsum(seq.DUR)])


def get_adc_sampling_times(seq) -> np.ndarray:
    """Sequence times of every ADC sample, in block order."""
    if isinstance(seq, HO_Sequence):
        seq = seq.simulation_sequence()
    starts = get_block_start_times(seq)
    out = [starts[j] + seq.ADC[j].times() for j in range(len(seq)) if seq.ADC[j].N > 0]
    return np.concatenate(out) if out else np.zeros(0)


def get_adc_phase_compensation(seq) -> np.ndarray:
    """exp(-i phi) of each ADC sample as single-precision complex numbers."""
    if isinstance(seq, HO_Sequence):
        seq = seq.SEQ
    out = [np.full(a.N, np.exp(-1j * a.phi), dtype=np.complex64) for a in seq.ADC if a.N > 0]
    return np.concatenate(out) if out else np.zeros(0, dtype=np.complex64)


def rf_pulses(seq, gamma: float = GAMMA):
    """(sequence time of the centre, flip angle in degrees) of every RF pulse
    that is on, in block order."""
    if isinstance(seq, HO_Sequence):
        seq = seq.simulation_sequence()
    starts = get_block_start_times(seq)
    out = []
    for j in range(len(seq)):
        rf = seq.RF[0, j]
        if rf.is_on():
            out.append((starts[j] + rf.center_time(), rf.flip_angle(gamma)))
    return out


# --------------------------------------------------------------------------- sampling

def _clusters(values: np.ndarray) -> np.ndarray:
    """Sorted representatives: values within _TOL of a representative join it."""
    v = np.sort(values)
    reps = [v[0]]
    for x in v[1:]:
        if x - reps[-1] > _TOL:
            reps.append(x)
    return np.asarray(reps)


def _snap(x: np.ndarray, reps: np.ndarray) -> np.ndarray:
    return reps[np.clip(np.searchsorted(reps, x, side="right") - 1, 0, reps.shape[0] - 1)]


def _snap_near(x: np.ndarray, reps: np.ndarray) -> np.ndarray:
    """Times within _TOL of a representative take its value; others stay."""
    i = np.clip(np.searchsorted(reps, x, side="right") - 1, 0, reps.shape[0] - 1)
    out = np.asarray(x, dtype=np.float64).copy()
    lo = np.abs(x - reps[i]) <= _TOL
    out[lo] = reps[i][lo]
    j = np.minimum(i + 1, reps.shape[0] - 1)
    hi = ~lo & (np.abs(reps[j] - x) <= _TOL)
    out[hi] = reps[j][hi]
    return out


def _right(tk, ak, q):
    """Right limits of the piecewise-linear waveform (tk, ak) at q (0 outside)."""
    k = np.searchsorted(tk, q, side="right") - 1
    out = np.zeros(q.shape[0], dtype=ak.dtype)
    ok = (k >= 0) & (k < tk.shape[0] - 1)
    k = k[ok]
    frac = (q[ok] - tk[k]) / (tk[k + 1] - tk[k])
    out[ok] = ak[k] + (ak[k + 1] - ak[k]) * frac
    return out


def _left(tk, ak, q):
    """Left limits of the waveform at q (0 outside)."""
    k = np.searchsorted(tk, q, side="left")
    out = np.zeros(q.shape[0], dtype=ak.dtype)
    ok = (k > 0) & (k < tk.shape[0])
    kk = k[ok]
    qq = q[ok]
    exact = tk[kk] == qq
    frac = np.where(exact, 1.0, (qq - tk[kk - 1]) / np.where(exact, 1.0, tk[kk] - tk[kk - 1]))
    val = ak[kk - 1] + (ak[kk] - ak[kk - 1]) * frac
    out[ok] = np.where(exact, ak[kk], val)
    return out


class _Block:
    __slots__ = ("t", "dt", "g", "h", "b1", "df", "adc", "exc")


def _sample_block(seq: Sequence, gr_dfc_col, j: int, rule: MaxStepSizeRule) -> _Block:
    D = float(seq.DUR[j])
    waves = [seq.GR[i, j] for i in range(3)] + list(gr_dfc_col)
    rf, adc = seq.RF[0, j], seq.ADC[j]
    rf_on = rf.is_on()
    knots = [w.knots() if w.is_on() else None for w in waves]
    keep = rule.preserve_samples
    raw = [np.array([0.0, D]), adc.times()] + [k[0] for k in knots[3:] if k is not None]
    if "gradients" in keep:
        raw += [k[0] for k in knots[:3] if k is not None]
    if rf_on:
        rk = rf.knots()
        raw.append(rk[0][[0, -1]])
        if "rf_center" in keep:
            raw.append(np.array([rf.center_time()]))
        if "rf" in keep:
            raw.append(rk[0])
    reps = _clusters(np.concatenate(raw))
    knots = [None if k is None else (_snap_near(k[0], reps), k[1]) for k in knots]
    if rf_on:
        rk = (_snap_near(rk[0], reps), rk[1])
        rf_s, rf_e = rk[0][0], rk[0][-1]

    # uniform fill between breakpoints
    a, b = reps[:-1], reps[1:]
    if a.shape[0]:
        lim = np.full(a.shape[0], rule.dt)
        if rf_on:
            mid = (a + b) / 2
            lim[(mid > rf_s) & (mid < rf_e)] = min(rule.dt, rule.dt_rf)
        cnt = np.maximum(1, np.ceil((b - a) / lim * (1 - 1e-9))).astype(np.int64)
        seg = np.repeat(np.arange(a.shape[0]), cnt)
        k = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        times = np.append(a[seg] + (b - a)[seg] * (k / cnt[seg]), reps[-1])
        is_bp = np.append(k == 0, True)
    else:
        times, is_bp = reps.copy(), np.ones(1, bool)

    # jumps of gradient / field waveforms at breakpoints
    bp = times[is_bp]
    jump_bp = np.zeros(bp.shape[0], bool)
    right = [None] * 19
    left_bp = [None] * 19
    for i, kn in enumerate(knots):
        if kn is None:
            continue
        right[i] = _right(kn[0], kn[1], times)
        left_bp[i] = _left(kn[0], kn[1], bp)
        jump_bp |= left_bp[i] != right[i][is_bp]
    dup = np.zeros(times.shape[0], bool)
    dup[np.flatnonzero(is_bp)[jump_bp]] = True
    src = np.repeat(np.arange(times.shape[0]), 1 + dup)
    n = src.shape[0]
    is_left = np.zeros(n, bool)
    starts_of = np.cumsum(1 + dup) - (1 + dup)
    is_left[starts_of[dup]] = True
    bp_index = np.full(times.shape[0], -1)
    bp_index[is_bp] = np.arange(bp.shape[0])

    out = _Block()
    out.t = times[src]
    vals = np.zeros((19, n))
    for i in range(19):
        if right[i] is None:
            continue
        v = right[i][src]
        li = np.flatnonzero(is_left)
        v[li] = left_bp[i][bp_index[src[li]]]
        vals[i] = v
    out.g, out.h = vals[:3], vals[3:]
    out.b1 = np.zeros(n, np.complex128)
    out.df = np.zeros(n)
    if rf_on:
        rr = _right(rk[0], rk[1], out.t)
        li = np.flatnonzero(is_left)
        if li.shape[0]:
            rr[li] = _left(rk[0], rk[1], out.t[li])
        out.b1 = rr
        inside = np.where(is_left, (out.t > rf_s) & (out.t <= rf_e), (out.t >= rf_s) & (out.t < rf_e))
        out.df = np.where(inside, rf.df, 0.0)
    out.dt = np.diff(out.t)
    out.adc = np.zeros(n, bool)
    if adc.N:
        at = _snap(adc.times(), reps)
        out.adc[np.searchsorted(out.t, at, side="right") - 1] = True
    if rf_on:
        out.exc = (out.dt > 0) & (out.t[:-1] >= rf_s) & (out.t[1:] <= rf_e)
    else:
        out.exc = np.zeros(max(n - 1, 0), bool)
    return out


class _Joiner:
    """Block concatenation with the boundary rule of HO_DiscreteSequence.jl:98-131."""

    def __init__(self):
        self.parts: List[dict] = []
        self.last = None  # (t, g, h, b1, df, adc) of the last node so far
        self.nnodes = 0

    def _push(self, t, dt, g, h, b1, df, adc, exc):
        self.parts.append(dict(t=t, dt=dt, g=g, h=h, b1=b1, df=df, adc=adc, exc=exc))
        self.last = (t[-1], g[:, -1].copy(), h[:, -1].copy(), b1[-1], df[-1], bool(adc[-1]))
        self.nnodes += t.shape[0]

    def append(self, blk: _Block, t0: float):
        first_t = t0 + blk.t[0]
        first = 0
        junction = None
        if self.last is None:
            if blk.adc[0]:  # keep an ADC sample on the very first node: pad in front of it
                z = np.zeros(1)
                self._push(np.array([first_t]), z[:0], blk.g[:, :1], blk.h[:, :1], blk.b1[:1], blk.df[:1],
                           np.zeros(1, bool), np.zeros(0, bool))
                junction = 0.0
        else:
            lt, lg, lh, lb1, ldf, ladc = self.last
            if abs(first_t - lt) <= _TOL * max(1.0, abs(lt)):
                first_t = lt
            if (first_t == lt and np.array_equal(lg, blk.g[:, 0]) and np.array_equal(lh, blk.h[:, 0])
                    and lb1 == blk.b1[0] and ldf == blk.df[0] and ladc == bool(blk.adc[0])):
                first = 1
            else:
                junction = max(first_t - lt, 0.0)
        t = t0 + blk.t[first:]
        if t.shape[0] == 0:
            return
        if first == 0:
            t[0] = first_t
        dt, exc = blk.dt, blk.exc  # a merged first node still opens the block's first interval
        if junction is not None:
            dt = np.concatenate([[junction], dt])
            exc = np.concatenate([[False], exc])
        self._push(t, dt, blk.g[:, first:], blk.h[:, first:], blk.b1[first:], blk.df[first:], blk.adc[first:], exc)

    def finish(self) -> HO_DiscreteSequence:
        cat = lambda k, ax=0: np.concatenate([p[k] for p in self.parts], axis=ax)  # noqa: E731
        g = cat("g", 1)
        return HO_DiscreteSequence(cat("t"), dt=cat("dt"), gx=g[0], gy=g[1], gz=g[2], b1=cat("b1"), df=cat("df"),
                                   adc=cat("adc"), excitation=cat("exc"), h=cat("h", 1))


def _rule(sampling_params, sampling_rule) -> MaxStepSizeRule:
    if sampling_rule is not None:
        if not isinstance(sampling_rule, MaxStepSizeRule):
            raise ArgumentError("sampling_rule must be a MaxStepSizeRule.")
        return sampling_rule
    p = sampling_params or {}
    if "sampling_rule" in p:
        return _rule(None, p["sampling_rule"])
    return MaxStepSizeRule(p.get("Δt", p.get("dt", 1e-3)), p.get("Δt_rf", p.get("dt_rf", 5e-5)),
                           p.get("preserve_samples", ("gradients", "rf_center")))


def discretize(hoseq: HO_Sequence, sampling_params=None, sampling_rule: Optional[MaxStepSizeRule] = None,
               freq_in_phase=None) -> HO_DiscreteSequence:
    """Sample the native events and all sixteen field waveforms on one grid
    (``discretize``, HO_DiscreteSequence.jl:133-179).  ``sampling_params``
    may give ``"Δt"`` / ``"Δt_rf"`` (or ``"dt"`` / ``"dt_rf"``) or a
    ``"sampling_rule"``; an explicit ``sampling_rule`` takes precedence.
    The caller's sequence is not modified."""
    if not isinstance(hoseq, HO_Sequence):
        raise ArgumentError("discretize takes an HO_Sequence.")
    if sampling_params is not None and not isinstance(sampling_params, dict):
        raise ArgumentError("sampling_params must be a dictionary.")
    if freq_in_phase is None:
        freq_in_phase = (sampling_params or {}).get("freq_in_phase", False)
    if freq_in_phase:
        raise ArgumentError("freq_in_phase=true is not supported: RF frequency offsets are sampled as df.")
    validate_high_order_sequence(hoseq)
    rule = _rule(sampling_params, sampling_rule)
    seq = hoseq.simulation_sequence()
    starts = get_block_start_times(seq)
    join = _Joiner()
    # A block's samples depend only on its duration and events: blocks that
    # share their event objects (a Pulseq file's repeated ids) are sampled once.
    cache = {}
    for j in range(len(seq)):
        waves = list(seq.GR[:, j]) + list(hoseq.GR_dfc[:, j])
        rf, adc = seq.RF[0, j], seq.ADC[j]
        key = (float(seq.DUR[j]), tuple(id(w) if w.is_on() else None for w in waves),
               id(rf) if rf.is_on() else None, id(adc) if adc.N else None)
        blk = cache.get(key)
        if blk is None:
            blk = cache[key] = _sample_block(seq, hoseq.GR_dfc[:, j], j, rule)
        join.append(blk, float(starts[j]))
    return join.finish()
