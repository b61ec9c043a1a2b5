"""Host-side data model mirroring HighOrderMRISim.jl's types for the
BlochHighOrder path.

The engine consumes *sampled* sequences: KomaMRI's discretisation and
``get_sim_ranges`` (KomaMRIBase 0.15.2 / KomaMRICore 0.14.0, not vendored in
the reference) stay on the caller's side.  ``get_sim_ranges`` below is a
documented restatement of the block-planning contract the engine needs
(consecutive intervals with one excitation flag, cut to a maximum length,
adjacent blocks sharing a node), used for synthetic workloads.

Name mapping to the reference (Julia field -> attribute here):
``ρ -> rho``, ``Δw -> dw``, ``Δt -> dt``, ``Δf -> df``, ``ψ -> psi``,
``ADC -> adc``, ``excitation_bool -> excitation``, ``h0..h15 -> h[0..15]``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

# KomaMRIBase's gyromagnetic ratio for 1H (Hz/T).
GAMMA = 42.5774688e6

HO0, HO1, HO2, HO3, DW_EXCITATION, DW_PRECESSION = 1, 2, 4, 8, 16, 32


class ArgumentError(ValueError):
    """Invalid argument (Julia's ``ArgumentError`` in the reference)."""


class DimensionMismatch(ValueError):
    """Inconsistent array sizes (Julia's ``DimensionMismatch``)."""


class BlochHighOrder:
    """Simulation method for dynamic fields through third spatial order.

    Mirrors ``src/simulation/BlochHighOrder.jl:21-43``: a four-character
    binary order mask (zeroth to third order) plus the ΔB0 flags for
    excitation and precession.  First order, when enabled, *replaces* the
    nominal gradients during precession; RF excitation always uses nominal
    gradients.
    """

    __slots__ = ("ho0", "ho1", "ho2", "ho3", "dw_excitation", "dw_precession", "name")

    def __init__(self, mask: str = "1111", dw_excitation: bool = True, dw_precession: bool = True):
        if not isinstance(mask, str) or len(mask) != 4 or any(ch not in "01" for ch in mask):
            raise ArgumentError(
                "The field-order mask must contain four binary digits, from order zero to three.")
        self.ho0, self.ho1, self.ho2, self.ho3 = (ch == "1" for ch in mask)
        self.dw_excitation = bool(dw_excitation)
        self.dw_precession = bool(dw_precession)
        self.name = mask

    @classmethod
    def from_flags(cls, ho0=True, ho1=True, ho2=True, ho3=True, dw_excitation=True, dw_precession=True,
                   name=None):
        expected = "".join("1" if bool(f) else "0" for f in (ho0, ho1, ho2, ho3))
        if name is not None and name != expected:
            raise ArgumentError("The field-order name must match ho0 through ho3.")
        return cls(expected, dw_excitation, dw_precession)

    @property
    def flags(self) -> int:
        return ((HO0 if self.ho0 else 0) | (HO1 if self.ho1 else 0) | (HO2 if self.ho2 else 0) |
                (HO3 if self.ho3 else 0) | (DW_EXCITATION if self.dw_excitation else 0) |
                (DW_PRECESSION if self.dw_precession else 0))

    def __repr__(self):
        return (f"BlochHighOrder[[{self.name}] zero order={self.ho0} | first order={self.ho1} | "
                f"second order={self.ho2} | third order={self.ho3} | Δw_excitation={self.dw_excitation} | "
                f"Δw_precession={self.dw_precession}]")

    def __eq__(self, other):
        return isinstance(other, BlochHighOrder) and self.flags == other.flags


class Bloch:
    """KomaMRICore's ``Bloch()`` on an ``HO_Phantom`` (accepted beside
    ``BlochHighOrder`` by setup_simulation, Simulate.jl:85-86): the nominal
    gradients and the off-resonance in both excitation and precession, no
    measured fields -- the same physics as ``BlochHighOrder("0000")``."""

    flags = DW_EXCITATION | DW_PRECESSION

    def __repr__(self):
        return "Bloch()"

    def __eq__(self, other):
        return isinstance(other, Bloch)

    def __hash__(self):
        return hash("Bloch")


def _vec(a, n, default, dtype):
    if a is None:
        return np.full(n, default, dtype=dtype)
    return np.asarray(a, dtype=dtype)


_SPIN_FIELDS = ("x", "y", "z", "rho", "T1", "T2", "T2s", "dw", "Dlambda1", "Dlambda2", "Dtheta")
_MOTION = ("ux", "uy", "uz")


def no_displacement(x, y, z, t):
    """The static phantom's displacement (HO_Phantom.jl:1)."""
    return 0


class HO_Phantom:
    """Spin phantom with receive sensitivities (``src/datatypes/HO_Phantom.jl:47-71``).

    Omitting ``csm`` gives one ideal receive coil with sensitivity ``1+0j`` at
    every spin.  Positions in metres, T1/T2 in seconds, ``dw`` in rad/s.  The
    diffusion parameters ``Dlambda1``, ``Dlambda2``, ``Dtheta`` (Julia's Dλ1,
    Dλ2, Dθ) are carried along and not used by BlochHighOrder.  ``ux``, ``uy``,
    ``uz`` are displacement functions f(x, y, z, t); the engine's kernels, like
    the reference's, need static coordinates (``no_displacement``).  ``a + b``
    concatenates spins (non-empty phantoms must share their displacement
    functions), ``alpha * obj`` scales the proton density only
    (HO_Phantom.jl:181-233).
    """

    def __init__(self, x, y=None, z=None, rho=None, T1=None, T2=None, T2s=None, dw=None, csm=None,
                 name="spins", dtype=np.float64, Dlambda1=None, Dlambda2=None, Dtheta=None,
                 ux=no_displacement, uy=no_displacement, uz=no_displacement):
        for f in (ux, uy, uz):
            if not callable(f):
                raise ArgumentError("ux, uy and uz must be functions of (x, y, z, t).")
        self.ux, self.uy, self.uz = ux, uy, uz
        x = np.asarray(x, dtype=dtype)
        n = x.shape[0] if x.ndim else 1
        self.name = name
        self.x = x.reshape(n)
        self.y = _vec(y, n, 0.0, dtype)
        self.z = _vec(z, n, 0.0, dtype)
        self.rho = _vec(rho, n, 1.0, dtype)
        self.T1 = _vec(T1, n, 1_000_000.0, dtype)
        self.T2 = _vec(T2, n, 1_000_000.0, dtype)
        self.T2s = _vec(T2s, n, 1_000_000.0, dtype)
        self.dw = _vec(dw, n, 0.0, dtype)
        self.Dlambda1 = _vec(Dlambda1, n, 0.0, dtype)
        self.Dlambda2 = _vec(Dlambda2, n, 0.0, dtype)
        self.Dtheta = _vec(Dtheta, n, 0.0, dtype)
        cdt = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
        # Column-major, as the reference's Julia arrays and the C ABI: the
        # array crosses to libhoms without a per-call transpose.
        if csm is None:
            self.csm = np.ones((n, 1), dtype=cdt, order="F")
        else:
            c = np.asarray(csm, dtype=cdt)
            self.csm = np.asfortranarray(c.reshape(c.shape[0], -1) if c.ndim == 1 else c)

    def __len__(self):
        return int(self.rho.shape[0])

    @property
    def ncoils(self) -> int:
        return int(self.csm.shape[1]) if self.csm.ndim == 2 else 0

    def validate(self):
        """Storage checks of ``validate_phantom`` (HO_Phantom.jl:97-109)."""
        n = len(self)
        for name in _SPIN_FIELDS:
            v = getattr(self, name)
            if v.ndim != 1 or v.shape[0] != n:
                raise DimensionMismatch(f"Phantom field {name} must contain one value per spin.")
        if self.csm.ndim != 2 or self.csm.shape[0] != n:
            raise DimensionMismatch("The CSM must have one row per spin.")

    def __getitem__(self, idx):
        if isinstance(idx, slice) or (isinstance(idx, np.ndarray) and idx.ndim == 1) or isinstance(idx, list):
            sl = idx
        else:
            sl = slice(int(idx), int(idx) + 1)
        out = HO_Phantom.__new__(HO_Phantom)
        out.name = self.name
        for k in _SPIN_FIELDS:
            setattr(out, k, getattr(self, k)[sl])
        for k in _MOTION:
            setattr(out, k, getattr(self, k))
        out.csm = self.csm[sl]
        return out

    def astype(self, dtype):
        out = HO_Phantom.__new__(HO_Phantom)
        out.name = self.name
        for k in _SPIN_FIELDS:
            setattr(out, k, np.asarray(getattr(self, k), dtype=dtype))
        for k in _MOTION:
            setattr(out, k, getattr(self, k))
        out.csm = np.asfortranarray(self.csm, dtype=np.complex64 if np.dtype(dtype) == np.float32 else np.complex128)
        return out

    def __repr__(self):
        ns, nc = self.csm.shape
        head = f"HO_Phantom[{self.name} | nCoil={nc} | nSpin={ns} | "
        if self.x.shape[0] == 0:
            return head + "empty ]"

        def span(v):
            lo, hi = (round(float(f) * 1e2, 2) for f in (np.min(v), np.max(v)))
            return f"{lo}:{hi} cm"
        return head + f"x={span(self.x)} | y={span(self.y)} | z={span(self.z)} ]"

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]

    def __add__(self, other: "HO_Phantom") -> "HO_Phantom":
        self.validate()
        other.validate()
        if self.ncoils != other.ncoils:
            raise DimensionMismatch("Concatenated phantoms must have the same number of receive coils.")
        if len(self) and len(other) and not all(getattr(self, k) is getattr(other, k) for k in _MOTION):
            raise ArgumentError("Cannot concatenate phantoms with different motion functions.")
        motion = other if len(self) == 0 else self
        out = HO_Phantom.__new__(HO_Phantom)
        out.name = f"{self.name}+{other.name}"
        for k in _MOTION:
            setattr(out, k, getattr(motion, k))
        for k in _SPIN_FIELDS:
            setattr(out, k, np.concatenate([getattr(self, k), getattr(other, k)]))
        out.csm = np.asfortranarray(np.concatenate([self.csm, other.csm], axis=0))
        return out

    def __mul__(self, alpha):
        if isinstance(alpha, (complex, np.complexfloating)) or not np.isscalar(alpha):
            return NotImplemented
        out = HO_Phantom.__new__(HO_Phantom)
        out.name = self.name
        for k in _SPIN_FIELDS:
            setattr(out, k, getattr(self, k))
        out.rho = alpha * self.rho
        for k in _MOTION:
            setattr(out, k, getattr(self, k))
        out.csm = self.csm
        return out

    def has_static_coordinates(self) -> bool:
        return all(getattr(self, k) is no_displacement for k in _MOTION)

    __rmul__ = __mul__

    def allclose(self, other: "HO_Phantom", rtol=1e-5, atol=1e-8) -> bool:
        """Field-wise closeness, as ``isapprox`` of two phantoms (HO_Phantom.jl:112-126)."""
        return (len(self) == len(other) and self.csm.shape == other.csm.shape
                and all(np.allclose(getattr(self, k), getattr(other, k), rtol=rtol, atol=atol) for k in _SPIN_FIELDS)
                and np.allclose(self.csm, other.csm, rtol=rtol, atol=atol))


class HO_DiscreteSequence:
    """Sampled sequence plus sixteen field-coefficient vectors
    (``src/datatypes/HO_DiscreteSequence.jl:31-80``).

    Node arrays have length Nt: ``t, gx, gy, gz, b1 (complex), df, psi, adc``
    and ``h`` (16 x Nt).  Interval arrays have length Nt-1: ``dt`` and
    ``excitation``.
    """

    def __init__(self, t, dt=None, gx=None, gy=None, gz=None, b1=None, df=None, psi=None, adc=None,
                 excitation=None, h=None, dtype=np.float64):
        t = np.asarray(t, dtype=dtype)
        nt = t.shape[0]
        self.t = t
        self.dt = np.diff(t) if dt is None else np.asarray(dt, dtype=dtype)
        self.gx = _vec(gx, nt, 0.0, dtype)
        self.gy = _vec(gy, nt, 0.0, dtype)
        self.gz = _vec(gz, nt, 0.0, dtype)
        cdt = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
        self.b1 = _vec(b1, nt, 0.0, cdt)
        self.df = _vec(df, nt, 0.0, dtype)
        self.psi = _vec(psi, nt, 0.0, dtype)
        self.adc = _vec(adc, nt, False, bool)
        self.excitation = _vec(excitation, max(nt - 1, 0), False, bool)
        if h is None:
            self.h = np.zeros((16, nt), dtype=dtype)
        else:
            h = np.asarray(h, dtype=dtype)
            self.h = h.reshape(16, nt)

    def __len__(self):
        """Number of intervals (KomaMRI's ``length(seqd)``)."""
        return int(self.dt.shape[0])

    @property
    def nnodes(self) -> int:
        return int(self.t.shape[0])

    def view(self, first: int, last: int) -> "HO_DiscreteSequence":
        """Nodes first..last inclusive (``Base.view(hoseqd, nodes)``, HO_DiscreteSequence.jl:73-76)."""
        out = HO_DiscreteSequence.__new__(HO_DiscreteSequence)
        sl = slice(first, last + 1)
        for k in ("t", "gx", "gy", "gz", "b1", "df", "psi", "adc"):
            setattr(out, k, getattr(self, k)[sl])
        out.dt = self.dt[first:last]
        out.excitation = self.excitation[first:last]
        out.h = self.h[:, sl]
        return out

    def astype(self, dtype):
        out = HO_DiscreteSequence.__new__(HO_DiscreteSequence)
        cdt = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
        for k in ("t", "dt", "gx", "gy", "gz", "df", "psi", "h"):
            setattr(out, k, np.asarray(getattr(self, k), dtype=dtype))
        out.b1 = np.asarray(self.b1, dtype=cdt)
        out.adc = self.adc.copy()
        out.excitation = self.excitation.copy()
        return out

    def validate(self):
        nt = self.nnodes
        if nt < 2:
            raise ArgumentError("The sequence must contain a simulation interval.")
        for k in ("gx", "gy", "gz", "b1", "df", "psi", "adc"):
            if getattr(self, k).shape != (nt,):
                raise DimensionMismatch(f"Sequence field {k} must contain one value per node.")
        if self.dt.shape != (nt - 1,) or self.excitation.shape != (nt - 1,):
            raise DimensionMismatch("Interval arrays must contain one value per interval.")
        if self.h.shape != (16, nt):
            raise DimensionMismatch("Each field coefficient must contain one value per node.")
        if np.any(np.asarray(self.dt) < 0):
            raise ArgumentError("Sampling intervals must be nonnegative.")


def get_sim_ranges(seqd: HO_DiscreteSequence, max_block_length=math.inf, max_rf_block_length=math.inf
                   ) -> Tuple[List[Tuple[int, int]], List[bool]]:
    """Plan time blocks over a sampled sequence.

    Restates the contract of KomaMRICore's ``get_sim_ranges`` as used by the
    reference (``src/simulation/Simulate.jl:116-123``): every block is a run of
    consecutive intervals sharing one excitation flag, at most
    ``max_block_length`` (``max_rf_block_length`` for RF) intervals long;
    adjacent blocks share their boundary node, whose ADC belongs to the
    earlier block.  Returns 0-based inclusive node ranges and flags.
    """
    for key, lim in (("max_block_length", max_block_length), ("max_rf_block_length", max_rf_block_length)):
        if not (lim == math.inf or (isinstance(lim, (int, np.integer)) and not isinstance(lim, bool) and lim > 0)):
            raise ArgumentError(f"{key} must be a positive integer or Inf.")
    exc = np.asarray(seqd.excitation, dtype=bool)
    n = exc.shape[0]
    parts: List[Tuple[int, int]] = []
    flags: List[bool] = []
    i = 0
    while i < n:
        flag = bool(exc[i])
        j = i
        while j < n and bool(exc[j]) == flag:
            j += 1
        lim = max_rf_block_length if flag else max_block_length
        k = i
        while k < j:
            e = j if lim == math.inf else min(j, k + int(lim))
            parts.append((k, e))
            flags.append(flag)
            k = e
        i = j
    return parts, flags


def count_block_adc(adc, parts: Sequence[Tuple[int, int]]) -> List[int]:
    """ADC samples per block: ADC[first+1 .. last] (SimulatorCore.jl:115-116)."""
    adc = np.asarray(adc, dtype=bool)
    return [int(adc[f + 1:l + 1].sum()) for f, l in parts]


@dataclass
class Mag:
    """Spin state: transverse ``xy`` (complex) and longitudinal ``z``."""
    xy: np.ndarray
    z: np.ndarray = field(default=None)


def initialize_spins_state(obj: HO_Phantom) -> Mag:
    """Mxy = 0, Mz = rho (``BlochHighOrderSimulatitonMethod.jl:9-15``)."""
    cdt = np.complex64 if obj.rho.dtype == np.float32 else np.complex128
    return Mag(np.zeros(len(obj), dtype=cdt), obj.rho.copy())


def rf_events(seqd: HO_DiscreteSequence, gamma: float = GAMMA, skip_rf=None):
    """RF breaks of a sampled sequence for the encoding export.

    The reference takes them from KomaMRIBase.get_RF_types on the unsampled
    sequence (``src/datatypes/HO_Sequence.jl:263``): every RF pulse cuts the
    k-space integral at its centre and is an excitation (flip angle up to
    90.01 degrees; the integral restarts) or a refocusing pulse (the integral
    changes sign).  Here a pulse is a run of consecutive excitation intervals
    with nonzero B1; its flip angle is 360 gamma sum |B1[n]| dt[n] degrees, its
    centre the |B1|-weighted mean interval midpoint, and its break the first
    interval of the run that starts at or after that centre.  ``skip_rf``
    (one flag per pulse) keeps the integral running through a pulse, as in
    the reference (:272).  Returns 0-based ``(rf_start, rf_sign)`` lists.
    """
    exc = np.asarray(seqd.excitation, dtype=bool)
    t = np.asarray(seqd.t, dtype=np.float64)
    dt = np.asarray(seqd.dt, dtype=np.float64)
    b1 = np.abs(np.asarray(seqd.b1, dtype=np.complex128))
    m = exc.shape[0]
    pulses = []
    i = 0
    while i < m:
        if not (exc[i] and b1[i] > 0):
            i += 1
            continue
        j = i
        while j < m and exc[j] and b1[j] > 0:
            j += 1
        w = b1[i:j] * dt[i:j]
        area = float(w.sum())
        centre = float((w * (t[i:j] + dt[i:j] / 2)).sum() / area) if area > 0 else float(t[i])
        start = next((n for n in range(i, j) if t[n] >= centre), j - 1)
        pulses.append((start, 360.0 * gamma * area))
        i = j
    return rf_break_lists(pulses, skip_rf, m)


def rf_break_lists(pulses, skip_rf, m: int):
    """``(rf_start, rf_sign)`` from ``(break interval, flip angle)`` per RF
    pulse over ``m`` intervals (``grad2kspace``, HO_Sequence.jl:262-279)."""
    if skip_rf is None:
        skip_rf = [False] * len(pulses)
    if len(skip_rf) != len(pulses):
        raise DimensionMismatch("skip_rf must contain one flag per RF event.")
    # As in the reference, part r + 1 takes the type of the r-th pulse
    # whichever break opened it; a break at the first interval opens no part
    # (kfoldperm's breaks are part starts).
    signs = [1 if skip else (0 if flip <= 90.01 else -1) for (_, flip), skip in zip(pulses, skip_rf)]
    rf_start = sorted({start for start, _ in pulses if 1 <= start < m})
    return rf_start, signs[:len(rf_start)]

