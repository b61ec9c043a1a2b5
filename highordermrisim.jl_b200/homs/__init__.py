"""homs -- host side of the B200 BlochHighOrder engine (libhoms).

Mirrors HighOrderMRISim.jl's simulation interface for the BlochHighOrder path:

* ``simulate(obj, seqd, sys=None, sim_params=...)`` -- one-shot simulation
  (``src/simulation/Simulate.jl:52-67`` / ``:204-219``);
* ``prepare_simulation(...)`` / ``Plan.run()`` / ``Plan.close()`` -- resident
  inputs reused across runs (``src/simulation/PreparedSimulation.jl:144-258``);
* the sampled-sequence and phantom containers, ``BlochHighOrder``, ``Bloch``
  and ``get_sim_ranges`` (see ``model``);
* event-level sequences (``Grad``, ``RF``, ``ADC``, ``Sequence``,
  ``HO_Sequence``) and ``discretize`` (see ``sequence``), Pulseq 1.4 files
  (``read_seq``) and the reference's demo inputs (``demo_inputs``; the
  timed demo workloads are ``bench_demo.py`` beside ``bench.py``);
* the encoding export ``get_kspace``, the phantom builders
  (``brain_phantom``, ``hophantom_brain``, ``csm_birdcage``, ``generate_grid``,
  ``Grid``), ``basisfunc_spha`` and the trajectory utilities;
* ``Server``, the continuous-batching front end, and ``ResidentPhantom``.

Every run executes in libhoms.so (sm_100a CUDA kernels).  There is no CPU
fallback: without the library or a B200 the calls raise ``HomsError``.
"""
from __future__ import annotations

import copy
import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Any, Dict, List, NamedTuple, Optional, Tuple

import numpy as np

from . import _lib
from ._lib import Context, HomsError
from .model import (GAMMA, ArgumentError, Bloch, BlochHighOrder, DimensionMismatch, HO_DiscreteSequence, HO_Phantom,
                    Mag, count_block_adc, get_sim_ranges, initialize_spins_state, rf_break_lists, rf_events)
from .sequence import (ADC, RF, Grad, HO_Sequence, MaxStepSizeRule, Sequence, discretize, get_adc_phase_compensation,
                       get_adc_sampling_times, get_block_start_times, rf_pulses)

__all__ = [
    "simulate", "prepare_simulation", "Plan", "Server", "Context", "HomsError", "ArgumentError", "DimensionMismatch",
    "BlochHighOrder", "HO_Phantom", "HO_DiscreteSequence", "Mag", "get_sim_ranges", "count_block_adc",
    "initialize_spins_state", "GAMMA", "HIGH_ORDER_COIL_COMBINATIONS", "RawData", "run_blocks", "get_kspace",
    "rf_events", "ResidentPhantom", "brain_phantom", "csm_birdcage", "grad2traj", "traj2grad", "InterpTrajTime",
    "Grad", "RF", "ADC", "Sequence", "HO_Sequence", "MaxStepSizeRule", "discretize", "get_adc_sampling_times",
    "get_adc_phase_compensation", "get_block_start_times", "read_seq", "demo2d_sequence", "demo3d_sequence",
    "Progress", "SimulationBlocks", "BlockData", "Bloch", "basisfunc_spha", "generate_grid", "hophantom_brain", "Grid",
]

# Accepted for source compatibility; every choice runs the fused libhoms kernel
# (src/simulation/kernels/HighOrderGPU.jl:4).
HIGH_ORDER_COIL_COMBINATIONS = ("gemm", "reduction", "fused_warp", "fused_tiled")

_DEFAULTS = {
    "precision": "f32", "return_type": "mat", "Nthreads": 1, "implementation": "auto", "coil_combination": "gemm",
    "synchronization": "auto", "max_block_length": math.inf, "max_rf_block_length": math.inf,
    "homs_precision": "plain", "gamma": GAMMA, "gpu_device": 0,
}


@dataclass
class RawData:
    """Minimal raw-acquisition container: one profile (samples x coils) per
    block that acquires, plus the run's parameters (``return_type="raw"``)."""
    profiles: List[np.ndarray]
    params: Dict[str, Any] = field(default_factory=dict)


def _sampled(seq, sim_params):
    """(sampled sequence, ADC phase compensation or None, native ADC count or
    None).  An ``HO_Sequence`` is discretised with the sampling keys of
    ``sim_params`` (``"Δt"``, ``"Δt_rf"``, ``"sampling_rule"``), as
    ``setup_simulation`` does (Simulate.jl:100)."""
    if isinstance(seq, Sequence):
        seq = HO_Sequence(seq)  # a native sequence: no measured fields
    if not isinstance(seq, HO_Sequence):
        if not isinstance(seq, HO_DiscreteSequence):
            raise ArgumentError("The sequence must be a Sequence, an HO_Sequence or an HO_DiscreteSequence.")
        return seq, None, None
    if sim_params is not None and not isinstance(sim_params, dict):
        raise ArgumentError("sim_params must be a dictionary with string keys.")
    seqd = discretize(seq, sampling_params=sim_params or {})
    comp = get_adc_phase_compensation(seq)
    if np.all(comp == 1):
        comp = None
    return seqd, comp, int(sum(a.N for a in seq.SEQ.ADC))


def _setup(obj: HO_Phantom, seqd: HO_DiscreteSequence, sim_params, parts=None, excitation=None, native_adc=None):
    """Validation and block planning of ``setup_simulation`` (Simulate.jl:222-287)."""
    if sim_params is None:
        sim_params = {}
    if not isinstance(sim_params, dict) or not all(isinstance(k, str) for k in sim_params):
        raise ArgumentError("sim_params must be a dictionary with string keys.")
    params = dict(_DEFAULTS)
    params.update(sim_params)
    params.setdefault("sim_method", BlochHighOrder("1111"))
    if params["synchronization"] not in ("auto", "block"):
        raise ArgumentError("synchronization must be auto or block.")
    if params["implementation"] not in ("auto", "kernel", "homs", "array"):
        raise ArgumentError("implementation must be auto, array, or kernel.")
    if params["implementation"] == "array":
        raise ArgumentError("implementation=array selects the reference's CPU/array path; this engine runs only "
                            "the libhoms CUDA kernels.")
    if params["coil_combination"] not in HIGH_ORDER_COIL_COMBINATIONS:
        raise ArgumentError(f"Unknown coil_combination: {params['coil_combination']}.")
    method = params["sim_method"]
    if not isinstance(method, (BlochHighOrder, Bloch)):
        raise ArgumentError("HO_Phantom currently supports Bloch() and BlochHighOrder().")
    if params["return_type"] not in ("mat", "state", "raw"):
        raise ArgumentError("return_type must be mat, state, or raw.")
    if params["precision"] not in ("f32", "f64"):
        raise ArgumentError("The legacy high-order path supports f32 and f64 precision.")
    if params["homs_precision"] not in ("plain", "split"):
        raise ArgumentError("homs_precision must be plain or split.")
    nth = params["Nthreads"]
    if not (isinstance(nth, (int, np.integer)) and not isinstance(nth, bool) and nth > 0):
        raise ArgumentError("Nthreads must be a positive integer.")
    if not isinstance(obj, HO_Phantom):
        raise ArgumentError("obj must be an HO_Phantom.")
    obj.validate()
    if len(obj) == 0:
        raise ArgumentError("The phantom must contain at least one spin.")
    if not obj.has_static_coordinates():
        raise ArgumentError("Moving phantoms (ux, uy, uz) need the reference's array path; the libhoms kernels, "
                            "like the reference's CUDA kernels, simulate static coordinates.")
    if obj.ncoils < 1:
        raise ArgumentError("The CSM must contain at least one coil.")
    seqd.validate()
    if parts is None:
        if "Nblocks" in sim_params:
            nb = sim_params["Nblocks"]
            if not (isinstance(nb, (int, np.integer)) and not isinstance(nb, bool) and nb > 0):
                raise ArgumentError("Nblocks must be a positive integer.")
            legacy = max(1, -(-len(seqd) // nb))
            if "max_block_length" not in sim_params:
                params["max_block_length"] = legacy
            if "max_rf_block_length" not in sim_params:
                params["max_rf_block_length"] = legacy
        parts, excitation = get_sim_ranges(seqd, params["max_block_length"], params["max_rf_block_length"])
    else:
        if excitation is None or len(excitation) != len(parts):
            raise DimensionMismatch("parts and excitation must have one entry per block.")
        parts = [(int(f), int(l)) for f, l in parts]
        excitation = [bool(e) for e in excitation]
    if not parts:
        raise ArgumentError("The sequence must contain a simulation interval.")
    if native_adc is not None and sum(count_block_adc(seqd.adc, parts)) != native_adc:
        raise DimensionMismatch("Sampled ADC count does not match the native sequence.")
    return params, parts, excitation


def _dtype(params):
    return _lib.HOMS_F64 if params["precision"] == "f64" else _lib.HOMS_F32


def _finalize(params, sig, state_xy, state_z, parts, excitation, seqd, seconds, comp=None):
    """finalize_simulation! (Simulate.jl:195-214).  ``comp`` is the ADC phase
    compensation of an event-level sequence (None: all ones)."""
    rt = params["return_type"]
    if rt == "state":
        return Mag(state_xy, state_z)
    if comp is not None and sig.shape[0]:
        # in place: sig is always this module's own freshly filled array
        np.multiply(sig, comp.astype(sig.dtype)[:, None], out=sig)
    if rt == "mat":
        return sig[:, :, None]
    counts = count_block_adc(seqd.adc, parts)
    profiles, k = [], 0
    for n in counts:
        if n:
            profiles.append(sig[k:k + n])
        k += n
    raw_params = {key: (str(v) if key == "sim_method" else v) for key, v in params.items()}
    raw_params.update({"Nblocks": len(parts), "type_sim_parts": list(excitation), "sim_time_sec": seconds})
    return RawData(profiles, raw_params)


def _state_arrays(obj, state, params, cdt, fdt):
    """(xy, z, pointer to the homs_state or None).  With no initial state and a
    return type that does not need the final one, no state crosses the ABI:
    the device starts from Mxy = 0, Mz = rho itself and keeps the result."""
    if state is None and params["return_type"] != "state":
        return None, None, None
    if state is None:
        xy = np.zeros(len(obj), dtype=cdt)
        z = np.ascontiguousarray(np.asarray(obj.rho, dtype=fdt)).copy()
    else:
        xy = np.ascontiguousarray(np.asarray(state.xy, dtype=cdt)).copy()
        z = np.ascontiguousarray(np.asarray(state.z, dtype=fdt)).copy()
    st = _lib.State(xy.ctypes.data, z.ctypes.data, _lib.HOMS_HOST)
    return xy, z, st


def _run_options(params) -> _lib.RunOptions:
    opts = _lib.RunOptions()
    opts.method = params["sim_method"].flags
    opts.mode = _lib.HOMS_SPLIT if params["homs_precision"] == "split" else _lib.HOMS_PLAIN
    return opts


_contexts: Dict[int, Context] = {}


def _context(device: int) -> Context:
    ctx = _contexts.get(device)
    if ctx is None or ctx.handle is None:
        ctx = Context(device)
        _contexts[device] = ctx
    return ctx


class ResidentPhantom:
    """A phantom kept on the device for many simulations (``homs_resident_*``).

    Its arrays are copied once, in the arithmetic's precision, and for
    ``homs_precision="split"`` its basis table and pre-split sensitivity
    operand are built once.  Pass it to ``simulate`` or ``Server.submit`` in
    place of the ``HO_Phantom``: only the sequence, the state and the signal
    move per simulation.  ``precision`` is the dtype the phantom arrives in
    and the results come back in.  Keep it open until every simulation that
    uses it has finished."""

    def __init__(self, obj: HO_Phantom, precision: str = "f64", homs_precision: str = "plain",
                 context: Optional[Context] = None):
        if not isinstance(obj, HO_Phantom):
            raise ArgumentError("obj must be an HO_Phantom.")
        if precision not in ("f32", "f64"):
            raise ArgumentError("The legacy high-order path supports f32 and f64 precision.")
        if homs_precision not in ("plain", "split"):
            raise ArgumentError("homs_precision must be plain or split.")
        obj.validate()
        self.obj, self.precision, self.homs_precision = obj, precision, homs_precision
        ctx = context or _context(0)
        self.device = ctx.device
        keep = _lib._Keep()
        ph = _lib.host_phantom(obj, keep, _lib.HOMS_F64 if precision == "f64" else _lib.HOMS_F32)
        mode = _lib.HOMS_SPLIT if homs_precision == "split" else _lib.HOMS_PLAIN
        h = ctypes.c_void_p()
        _lib.check(_lib.load().homs_resident_create(ctx.handle, ctypes.byref(ph), mode, ctypes.byref(h)), ctx.handle)
        self.handle = h

    def __len__(self):
        return len(self.obj)

    def device_bytes(self) -> int:
        n = ctypes.c_size_t()
        _lib.check(_lib.load().homs_resident_device_bytes(self.handle, ctypes.byref(n)))
        return int(n.value)

    def close(self):
        if self.handle is not None:
            _lib.load().homs_resident_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _resident_args(obj, sim_params):
    """(HO_Phantom, ResidentPhantom or None, sim_params) for a call given an
    HO_Phantom or a ResidentPhantom; a resident fixes precision and homs_precision."""
    sim_params = dict(sim_params or {})
    if not isinstance(obj, ResidentPhantom):
        return obj, None, sim_params
    if obj.handle is None:
        raise ArgumentError("The resident phantom is closed.")
    for key, val in (("precision", obj.precision), ("homs_precision", obj.homs_precision)):
        if sim_params.setdefault(key, val) != val:
            raise ArgumentError(f"{key} must be the resident phantom's ({val}).")
    return obj.obj, obj, sim_params


def simulate(obj: HO_Phantom, seqd: HO_DiscreteSequence = None, sys=None, *, sim_params=None, parts=None,
             excitation=None, state: Optional[Mag] = None, context: Optional[Context] = None, gpus=None, callbacks=(),
             verbose=False, return_type=None):
    """Simulate ``obj`` under ``seqd``: an ``HO_Sequence`` (discretised first,
    with the ``"Δt"`` / ``"Δt_rf"`` sampling keys of ``sim_params``, and its
    ADC phase compensation applied) or an already sampled
    ``HO_DiscreteSequence``.

    ``sim_params`` keys follow the reference: ``"sim_method"``
    (BlochHighOrder), ``"precision"`` (f32/f64), ``"return_type"``
    (mat/state/raw), ``"max_block_length"``, ``"max_rf_block_length"``,
    ``"Nblocks"``, plus ``"homs_precision"`` (``"plain"`` or ``"split"``).
    ``parts``/``excitation`` give KomaMRICore's block plan explicitly
    (0-based inclusive node ranges); by default ``get_sim_ranges`` plans it.
    ``sys`` (the KomaMRI Scanner) is accepted and unused, as in the reference
    path.  Returns (Nadc, Nc, 1) complex for "mat", ``Mag`` for "state".
    The caller's dictionary is never modified.

    ``callbacks`` (callables) are called after every block with
    ``(Progress, SimulationBlocks, BlockData, sim_params)``, as the
    reference's block loop calls them (SimulatorCore.jl:144-149); the blocks
    then run one at a time, each from the state the previous one left.

    ``simulate(plan, return_type=...)`` runs a prepared ``Plan`` instead
    (``simulate(plan::PreparedSimulation)``, PreparedSimulation.jl:218-258).
    """
    if isinstance(obj, Plan):
        if seqd is not None or sim_params is not None or parts is not None or state is not None:
            raise ArgumentError("A prepared simulation takes only return_type (and callbacks, verbose).")
        return obj.run(return_type, callbacks)
    if return_type is not None:
        raise ArgumentError("return_type is a sim_params key here; the keyword is for prepared simulations.")
    if seqd is None:
        raise ArgumentError("simulate needs a sequence (or a prepared simulation).")
    obj, resident, sim_params = _resident_args(obj, sim_params)
    seqd, comp, native_adc = _sampled(seqd, sim_params)
    params, parts, excitation = _setup(obj, seqd, sim_params, parts, excitation, native_adc)
    if gpus is not None:
        if not isinstance(gpus, (list, tuple)) or len(gpus) != 1 or not isinstance(gpus[0], (int, np.integer)) \
                or isinstance(gpus[0], bool) or gpus[0] < 0:
            raise ArgumentError("gpus must name exactly one visible device on this engine.")
        params["gpu_device"] = int(gpus[0])
    if resident is not None and gpus is None:
        params["gpu_device"] = resident.device
    ctx = context or _context(int(params["gpu_device"]))
    if callbacks:
        sig, cur, seconds = _run_with_callbacks(obj, seqd, params, parts, excitation, state, ctx, callbacks)
        return _finalize(params, sig, cur.xy, cur.z, parts, excitation, seqd, seconds, comp)
    dt = _dtype(params)
    keep = _lib._Keep()
    ph = _lib.host_phantom(obj, keep, dt) if resident is None else None
    sq = _lib.host_sequence(seqd, parts, excitation, keep, dt, params["gamma"])
    nadc = sum(count_block_adc(seqd.adc, parts))
    cdt = np.complex128 if dt == _lib.HOMS_F64 else np.complex64
    fdt = np.float64 if dt == _lib.HOMS_F64 else np.float32
    sig = np.zeros((nadc, obj.ncoils), dtype=cdt, order="F")
    xy, z, st = _state_arrays(obj, state, params, cdt, fdt)
    st_ref = ctypes.byref(st) if st is not None else None
    opts = _run_options(params)
    t0 = time.perf_counter()
    lib = _lib.load()
    if resident is None:
        _lib.check(lib.homs_simulate(ctx.handle, ctypes.byref(ph), ctypes.byref(sq), ctypes.byref(opts),
                                     st_ref, sig.ctypes.data if nadc else None, _lib.HOMS_HOST), ctx.handle)
    else:
        _lib.check(lib.homs_simulate_resident(ctx.handle, resident.handle, ctypes.byref(sq), ctypes.byref(opts),
                                              st_ref, sig.ctypes.data if nadc else None, _lib.HOMS_HOST),
                   ctx.handle)
    seconds = time.perf_counter() - t0
    return _finalize(params, np.asarray(sig), xy, z, parts, excitation, seqd, seconds, comp)


class Progress(NamedTuple):
    """``progress_info`` of the reference's block loop (SimulatorCore.jl:144):
    the block just finished (1-based), the number of blocks, RF blocks so far,
    and the 1-based index of the next ADC sample."""
    block: int
    Nblocks: int
    rfs: int
    samples: int


class SimulationBlocks(NamedTuple):
    """``simulation_blocks_info``: excitation flag and 0-based inclusive node range of every block."""
    excitation_bool: List[bool]
    parts: List[Tuple[int, int]]


class BlockData(NamedTuple):
    """``device_data`` after a block: phantom, sampled sequence, the signal so
    far (rows of later blocks still zero) and the spin state ``Xt``."""
    obj: Any
    seqd: Any
    sig: np.ndarray
    Xt: Mag


def _run_with_callbacks(obj, seqd, params, parts, excitation, state, ctx, callbacks):
    """The block loop of run_sim_time_iter! (SimulatorCore.jl:96-152) with its
    callbacks: each block runs on the device by itself, from the state the
    previous block left, and every callback is called after it with
    ``(Progress, SimulationBlocks, BlockData, sim_params)`` on completed data.
    The phantom and sequence the callbacks see are this run's copies; an edit
    to them or to the state reaches the following blocks of the run only."""
    for cb in callbacks:
        if not callable(cb):
            raise ArgumentError("callbacks must be callables.")
    # The run's own copies: a callback may edit them, and later blocks of this
    # run see the edits, as they see the reference's device copies.
    obj, seqd = copy.deepcopy(obj), copy.deepcopy(seqd)
    method, prec, mode = params["sim_method"], params["precision"], params["homs_precision"]
    cdt = np.complex128 if prec == "f64" else np.complex64
    fdt = np.float64 if prec == "f64" else np.float32
    nadc = sum(count_block_adc(seqd.adc, parts))
    sig = np.zeros((nadc, obj.ncoils), dtype=cdt, order="F")
    cur = state if state is not None else Mag(np.zeros(len(obj), cdt), np.asarray(obj.rho, fdt).copy())
    info = SimulationBlocks(list(excitation), list(parts))
    samples, rfs = 1, 0
    t0 = time.perf_counter()
    for b, ((f, l), e) in enumerate(zip(parts, excitation), start=1):
        blk, xy, z = run_blocks(obj, seqd.view(f, l), [(0, l - f)], [e], method, prec, mode, cur, ctx,
                                params["gamma"])
        sig[samples - 1:samples - 1 + blk.shape[0]] = blk
        samples += blk.shape[0]
        rfs += int(bool(e))
        cur = Mag(xy, z)
        progress = Progress(b, len(parts), rfs, samples)
        data = BlockData(obj, seqd, sig, cur)
        for cb in callbacks:
            cb(progress, info, data, params)
    return sig, cur, time.perf_counter() - t0


def run_blocks(obj: HO_Phantom, seqd: HO_DiscreteSequence, parts, excitation, method: BlochHighOrder,
               precision: str = "f64", mode: str = "plain", state: Optional[Mag] = None,
               context: Optional[Context] = None, gamma: float = GAMMA):
    """Run an explicit block plan and return ``(signal (Nadc x Nc), Mxy, Mz)``:
    the kernel-level counterpart of ``simulate_shard`` (Simulate.jl:138-193)."""
    if precision not in ("f32", "f64"):
        raise ArgumentError("precision must be f32 or f64")
    if mode not in ("plain", "split"):
        raise ArgumentError("mode must be plain or split")
    obj.validate()
    seqd.validate()
    ctx = context or _context(0)
    dt = _lib.HOMS_F64 if precision == "f64" else _lib.HOMS_F32
    keep = _lib._Keep()
    ph = _lib.host_phantom(obj, keep, dt)
    sq = _lib.host_sequence(seqd, parts, excitation, keep, dt, gamma)
    nadc = sum(count_block_adc(seqd.adc, parts))
    cdt = np.complex128 if dt == _lib.HOMS_F64 else np.complex64
    fdt = np.float64 if dt == _lib.HOMS_F64 else np.float32
    sig = np.zeros((nadc, obj.ncoils), dtype=cdt, order="F")
    if state is None:
        xy = np.zeros(len(obj), dtype=cdt)
        z = np.ascontiguousarray(np.asarray(obj.rho, dtype=fdt)).copy()
    else:
        xy = np.ascontiguousarray(np.asarray(state.xy, dtype=cdt)).copy()
        z = np.ascontiguousarray(np.asarray(state.z, dtype=fdt)).copy()
    st = _lib.State(xy.ctypes.data, z.ctypes.data, _lib.HOMS_HOST)
    opts = _lib.RunOptions()
    opts.method = method.flags if isinstance(method, (BlochHighOrder, Bloch)) else int(method)
    opts.mode = _lib.HOMS_SPLIT if mode == "split" else _lib.HOMS_PLAIN
    _lib.check(_lib.load().homs_simulate(ctx.handle, ctypes.byref(ph), ctypes.byref(sq), ctypes.byref(opts),
                                         ctypes.byref(st), sig.ctypes.data if nadc else None, _lib.HOMS_HOST),
               ctx.handle)
    return np.asarray(sig), xy, z


def _kspace_inputs(hoseq: HO_Sequence, dt, skip_rf, sampling_rule, gamma):
    """Sampled sequence, RF breaks and ADC times of an event-level sequence
    (HO_Sequence.jl:236-255): sampling at ``MaxStepSizeRule(dt, 5e-5)``, one
    break per RF pulse at the first node at or after its centre."""
    seqd = discretize(hoseq, sampling_rule=sampling_rule or MaxStepSizeRule(dt, 5e-5))
    t = np.asarray(seqd.t[:-1], dtype=np.float64)
    pulses = [(int(np.searchsorted(t, c - 1e-12 * max(1.0, abs(c)), side="left")), flip)
              for c, flip in rf_pulses(hoseq, gamma)]
    rf_start, rf_sign = rf_break_lists(pulses, skip_rf, t.shape[0])
    return seqd, rf_start, rf_sign, get_adc_sampling_times(hoseq)


def get_kspace(seqd, rf_start=None, rf_sign=None, skip_rf=None, adc_times=None,
               gamma: float = GAMMA, context: Optional[Context] = None, precision: str = "f64", dt=1.0,
               sampling_rule=None):
    """``K_nominal, K_nominal_adc, K_dfc, K_dfc_adc`` of a sequence on the GPU
    (``get_kspace``, src/datatypes/HO_Sequence.jl:236-255).

    An ``HO_Sequence`` is sampled first (``dt``, ``sampling_rule``), its RF
    pulses give the breaks and its ADC windows the ADC times.  For a sampled
    ``HO_DiscreteSequence`` the arguments below apply.

    ``K_nominal`` (Nt-1 x 3) integrates the nominal gradients and ``K_dfc``
    (Nt-1 x 16) the sixteen field coefficients, with KomaMRICore's cumtrapz,
    restarted or negated at the RF breaks; the ``_adc`` copies interpolate them
    at ``adc_times`` (default: the times of the ADC nodes).  The RF breaks are
    ``rf_start`` / ``rf_sign`` (0-based interval indices; 0 excitation, -1
    refocusing, +1 kept) or, by default, ``rf_events(seqd, gamma, skip_rf)``.
    ``precision`` is the dtype the sequence arrays cross the ABI in; the
    integral is FP64 either way."""
    if isinstance(seqd, Sequence):
        seqd = HO_Sequence(seqd)
    if isinstance(seqd, HO_Sequence):
        if rf_start is not None or rf_sign is not None or adc_times is not None:
            raise ArgumentError("rf_start, rf_sign and adc_times come from the HO_Sequence itself.")
        seqd, rf_start, rf_sign, adc_times = _kspace_inputs(seqd, dt, skip_rf, sampling_rule, gamma)
    seqd.validate()
    if rf_start is None:
        if rf_sign is not None:
            raise ArgumentError("rf_sign needs rf_start")
        rf_start, rf_sign = rf_events(seqd, gamma, skip_rf)
    elif rf_sign is None or len(rf_sign) != len(rf_start):
        raise DimensionMismatch("rf_sign must contain one value per RF break.")
    if precision not in ("f32", "f64"):
        raise ArgumentError("precision must be f32 or f64")
    if adc_times is None:
        adc_times = np.asarray(seqd.t, dtype=np.float64)[np.asarray(seqd.adc, dtype=bool)]
    ctx = context or _context(0)
    dt = _lib.HOMS_F64 if precision == "f64" else _lib.HOMS_F32
    keep = _lib._Keep()
    nt = seqd.nnodes
    sq = _lib.host_sequence(seqd, [(0, nt - 1)], [False], keep, dt, gamma)
    starts = np.ascontiguousarray(rf_start, dtype=np.int64)
    signs = np.ascontiguousarray(rf_sign, dtype=np.int8)
    q = np.ascontiguousarray(adc_times, dtype=np.float64)
    k = np.zeros((nt - 1, 19), order="F")
    kq = np.zeros((q.shape[0], 19), order="F")
    _lib.check(_lib.load().homs_kspace(ctx.handle, ctypes.byref(sq), len(starts),
                                       starts.ctypes.data if len(starts) else None,
                                       signs.ctypes.data if len(signs) else None, q.shape[0],
                                       q.ctypes.data if q.shape[0] else None, k.ctypes.data,
                                       kq.ctypes.data if q.shape[0] else None, _lib.HOMS_HOST), ctx.handle)
    return k[:, :3], kq[:, :3], k[:, 3:], kq[:, 3:]


class Plan:
    """Prepared simulation: inputs resident on the device, repeated runs
    restart from Mxy = 0, Mz = rho (PreparedSimulation.jl:144-258)."""

    def __init__(self, obj, seqd, sys=None, sim_params=None, parts=None, excitation=None,
                 context: Optional[Context] = None):
        seqd, self.comp, native_adc = _sampled(seqd, sim_params)
        params, parts, excitation = _setup(obj, seqd, dict(sim_params or {}), parts, excitation, native_adc)
        self.params = params
        self.parts, self.excitation = parts, excitation
        self.seqd = seqd
        self._host = copy.deepcopy(obj)  # snapshot for runs with callbacks (block by block)
        self._busy = False
        self.ctx = context or _context(int(params["gpu_device"]))
        self.dtype = _dtype(params)
        self.ns, self.nc = len(obj), obj.ncoils
        self.nadc = sum(count_block_adc(seqd.adc, parts))
        keep = _lib._Keep()
        ph = _lib.host_phantom(obj, keep, self.dtype)
        sq = _lib.host_sequence(seqd, parts, excitation, keep, self.dtype, params["gamma"])
        opts = _run_options(params)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().homs_plan_create(self.ctx.handle, ctypes.byref(ph), ctypes.byref(sq),
                                                ctypes.byref(opts), ctypes.byref(h)), self.ctx.handle)
        self.handle = h
        self.closed = False

    def run(self, return_type=None, callbacks=()):
        """One run from Mxy = 0, Mz = rho.  With ``callbacks`` the run goes block
        by block from the plan's snapshot of the phantom, calling each callback
        after every block as ``simulate`` does."""
        if return_type is None:
            return_type = self.params["return_type"]
        if return_type not in ("mat", "state", "raw"):
            raise ArgumentError("return_type must be mat, state, or raw.")
        if self._busy:
            raise ArgumentError("A prepared simulation cannot be used recursively from its callback.")
        if self.closed:
            raise ArgumentError("The prepared simulation is closed.")
        if callbacks:
            params = dict(self.params)
            params["return_type"] = return_type
            self._busy = True
            try:
                sig, cur, seconds = _run_with_callbacks(self._host, self.seqd, params, self.parts, self.excitation,
                                                        None, self.ctx, callbacks)
            finally:
                self._busy = False
            return _finalize(params, sig, cur.xy, cur.z, self.parts, self.excitation, self.seqd, seconds, self.comp)
        cdt = np.complex128 if self.dtype == _lib.HOMS_F64 else np.complex64
        fdt = np.float64 if self.dtype == _lib.HOMS_F64 else np.float32
        sig = np.zeros((self.nadc, self.nc), dtype=cdt, order="F")
        xy = z = st = None
        if return_type == "state":  # the final state is copied back only when it is returned
            xy = np.zeros(self.ns, dtype=cdt)
            z = np.zeros(self.ns, dtype=fdt)
            st = _lib.State(xy.ctypes.data, z.ctypes.data, _lib.HOMS_HOST)
        t0 = time.perf_counter()
        _lib.check(_lib.load().homs_plan_run(self.handle, sig.ctypes.data if self.nadc else None, _lib.HOMS_HOST,
                                             ctypes.byref(st) if st is not None else None), self.ctx.handle)
        params = dict(self.params)
        params["return_type"] = return_type
        return _finalize(params, np.asarray(sig), xy, z, self.parts, self.excitation, self.seqd,
                         time.perf_counter() - t0, self.comp)

    def device_bytes(self) -> int:
        n = ctypes.c_size_t()
        _lib.check(_lib.load().homs_plan_device_bytes(self.handle, ctypes.byref(n)))
        return int(n.value)

    def graph_state(self) -> Tuple[int, str]:
        """(1, "") while runs replay the plan's captured CUDA graph, (0, "")
        before the capture (the second run), (-1, reason) if capture failed
        and runs are issued kernel by kernel."""
        st, why = ctypes.c_int32(), ctypes.c_char_p()
        _lib.check(_lib.load().homs_plan_graph(self.handle, ctypes.byref(st), ctypes.byref(why)))
        return int(st.value), (why.value or b"").decode()

    def close(self):
        if self._busy:
            raise ArgumentError("A prepared simulation cannot be closed from its callback.")
        if not self.closed:
            _lib.load().homs_plan_destroy(self.handle)
            self.handle = None
            self.closed = True

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def prepare_simulation(obj, seqd, sys=None, *args, sim_params=None, parts=None, excitation=None, context=None):
    """Create a ``Plan`` (use as a context manager or call ``close()``).

    ``prepare_simulation(f, obj, seqd, ...)`` is the do-block form of
    PreparedSimulation.jl:181-188: it returns ``f(plan)`` and closes the plan
    whatever happens."""
    if callable(obj) and not isinstance(obj, (HO_Phantom, ResidentPhantom)):
        f, obj, seqd, sys = obj, seqd, sys, (args[0] if args else None)
        plan = Plan(obj, seqd, sys, sim_params, parts, excitation, context)
        try:
            return f(plan)
        finally:
            plan.close()
    if args:
        raise ArgumentError("prepare_simulation takes (obj, seqd, sys) or (f, obj, seqd, sys).")
    return Plan(obj, seqd, sys, sim_params, parts, excitation, context)


@dataclass
class _Request:
    keep: Any
    sig: np.ndarray
    xy: np.ndarray
    z: np.ndarray
    params: Dict[str, Any]
    parts: Any
    excitation: Any
    seqd: Any
    structs: Tuple[Any, ...]
    comp: Any = None


class Server:
    """Continuous-batching simulation server (``homs_server_*``).

    Requests run as ``simulate`` would run them, on ``slots`` concurrent
    contexts of one device; a request is admitted in submission order as soon
    as a slot is free and its device footprint fits in ``max_device_bytes``
    (0: three quarters of the free device memory) beside the requests in
    flight.  ``submit`` returns a ticket; ``result`` waits for it and returns
    what ``simulate`` returns.  The serving counterpart of the reference's
    persistent worker (src/simulation/PreparedSimulation.jl:2-287).
    """

    def __init__(self, device: int = 0, slots: int = 4, max_device_bytes: int = 0):
        self._lib = _lib.load()
        opts = _lib.ServerOptions()
        opts.device = int(device)
        opts.slots = int(slots)
        opts.max_device_bytes = int(max_device_bytes)
        h = ctypes.c_void_p()
        _lib.check(self._lib.homs_server_create(ctypes.byref(opts), ctypes.byref(h)))
        self.handle = h
        self._requests: Dict[int, _Request] = {}

    def submit(self, obj: HO_Phantom, seqd: HO_DiscreteSequence, *, sim_params=None, parts=None, excitation=None,
               state: Optional[Mag] = None) -> int:
        """Queue one simulation; the arguments are those of ``simulate`` (``obj``
        an ``HO_Phantom`` or a ``ResidentPhantom`` of the server's device)."""
        if self.handle is None:
            raise HomsError(6, "server is closed")
        obj, resident, sim_params = _resident_args(obj, sim_params)
        seqd, comp, native_adc = _sampled(seqd, sim_params)
        params, parts, excitation = _setup(obj, seqd, sim_params, parts, excitation, native_adc)
        dt = _dtype(params)
        keep = _lib._Keep()
        ph = _lib.host_phantom(obj, keep, dt) if resident is None else None
        sq = _lib.host_sequence(seqd, parts, excitation, keep, dt, params["gamma"])
        nadc = sum(count_block_adc(seqd.adc, parts))
        cdt = np.complex128 if dt == _lib.HOMS_F64 else np.complex64
        fdt = np.float64 if dt == _lib.HOMS_F64 else np.float32
        sig = np.zeros((nadc, obj.ncoils), dtype=cdt, order="F")
        xy, z, st = _state_arrays(obj, state, params, cdt, fdt)
        st_ref = ctypes.byref(st) if st is not None else None
        opts = _run_options(params)
        ticket = ctypes.c_int64()
        if resident is None:
            _lib.check(self._lib.homs_server_submit(self.handle, ctypes.byref(ph), ctypes.byref(sq),
                                                    ctypes.byref(opts), st_ref,
                                                    sig.ctypes.data if nadc else None, _lib.HOMS_HOST,
                                                    ctypes.byref(ticket)))
        else:
            _lib.check(self._lib.homs_server_submit_resident(self.handle, resident.handle, ctypes.byref(sq),
                                                             ctypes.byref(opts), st_ref,
                                                             sig.ctypes.data if nadc else None, _lib.HOMS_HOST,
                                                             ctypes.byref(ticket)))
        self._requests[ticket.value] = _Request(keep, sig, xy, z, params, parts, excitation, seqd,
                                                (ph, sq, st, opts, resident), comp)
        return ticket.value

    def done(self, ticket: int) -> bool:
        """True once the request has finished (successfully or not)."""
        return self._lib.homs_server_poll(self.handle, int(ticket)) != 7

    def times(self, ticket: int) -> Tuple[float, float, float]:
        """(submitted, started, finished) in seconds since the server started."""
        t = _lib.RequestTimes()
        self._lib.homs_server_times(self.handle, int(ticket), ctypes.byref(t))
        return t.submitted, t.started, t.finished

    def estimate(self, ticket: int) -> int:
        """The request's admission estimate of its device footprint in bytes."""
        b = ctypes.c_int64(0)
        _lib.check(self._lib.homs_server_estimate(self.handle, int(ticket), ctypes.byref(b)))
        return int(b.value)

    def result(self, ticket: int, timeout: float = 600.0):
        """Wait for a request and return what ``simulate`` returns for it."""
        req = self._requests[int(ticket)]
        status = self._lib.homs_server_wait(self.handle, int(ticket), float(timeout))
        if status != 0:
            msg = self._lib.homs_server_error(self.handle, int(ticket))
            raise HomsError(status, (msg or b"").decode() or _lib.load().homs_status_string(status).decode())
        t0, t1, t2 = self.times(ticket)
        # a copy when the phase compensation applies: result() may be asked again
        sig = np.array(req.sig) if req.comp is not None else np.asarray(req.sig)
        return _finalize(req.params, sig, req.xy, req.z, req.parts, req.excitation, req.seqd, t2 - t1, req.comp)

    def release(self, ticket: int) -> None:
        """Forget a finished request (its buffers are released)."""
        if self._lib.homs_server_release(self.handle, int(ticket)) == 0:
            self._requests.pop(int(ticket), None)

    def close(self) -> None:
        """Finish every queued request and free the server."""
        if self.handle is not None:
            self._lib.homs_server_destroy(self.handle)
            self.handle = None
            self._requests.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


from .phantom import Grid, brain_phantom, csm_birdcage, generate_grid, hophantom_brain  # noqa: E402
from .trajectory import InterpTrajTime, grad2traj, traj2grad  # noqa: E402
from .pulseq import read_seq  # noqa: E402
from .sphericalharmonics import basisfunc_spha  # noqa: E402
from .demo_inputs import demo2d_sequence, demo3d_sequence  # noqa: E402
