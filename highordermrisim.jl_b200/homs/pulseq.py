"""Pulseq 1.4 sequence files to event-level sequences.

The reference reads its demo sequences with KomaMRIFiles' ``read_seq``
(demo3D/1_load_seq.jl:14, demo2D/1_load_inputs.jl:42), a third-party package
that is not vendored.  This module restates the published Pulseq 1.4 file
format (sections ``[VERSION]``, ``[DEFINITIONS]``, ``[BLOCKS]``, ``[RF]``,
``[GRADIENTS]``, ``[TRAP]``, ``[ADC]``, ``[EXTENSIONS]``, ``[SHAPES]``,
``[SIGNATURE]``) and maps each event onto ``homs.sequence``:

* ``[TRAP]`` ``id amplitude rise flat fall delay`` (Hz/m, us) ->
  ``Grad(amplitude / gamma, flat, rise, fall, delay)``.
* ``[GRADIENTS]`` ``id amplitude amp_shape_id time_shape_id delay``: with
  time shape 0 the samples sit at (k + 1/2) gradient rasters, so the event
  is ``Grad(w, (n - 1) raster, raster / 2, raster / 2, delay)`` (the
  convention the reference's demo uses for its measured waveforms,
  demo3D/1_load_seq.jl:54-58); with a time shape (in rasters) the samples
  sit at those times and the waveform's first and last samples are its
  ``first`` and ``last``.
* ``[RF]`` ``id amplitude mag_id phase_id time_shape_id delay freq phase``:
  B1 = amplitude / gamma * mag * exp(i (2 pi phase_shape + phase)) (the phase
  shape is in turns), samples at (k + 1/2) RF rasters or at the time shape,
  frequency offset ``freq`` (Hz).
* ``[ADC]`` ``id num dwell delay freq phase`` (ns, us, Hz, rad): samples at
  ``delay + (k + 1/2) dwell`` -> ``ADC(num, (num - 1) dwell, delay + dwell/2,
  freq, phase)``.
* ``[BLOCKS]`` ``NUM DUR RF GX GY GZ ADC EXT``: DUR in block-duration
  rasters.  Extension lists (labels, triggers) are kept as ids and not
  interpreted: they do not change the simulated signal.
* ``[SHAPES]``: a shape listed with fewer values than ``num_samples`` is the
  run-length-encoded derivative (a value repeated twice is followed by the
  count of further repeats) and is integrated by a cumulative sum.

``[DEFINITIONS]`` become ``Sequence.DEF`` (numbers as floats or float
lists).  ``signature_ok`` checks the md5 of the file up to its signature.
"""
from __future__ import annotations

import hashlib
import math
from typing import Dict, List

import numpy as np

from .model import GAMMA, ArgumentError
from .sequence import ADC, RF, Grad, Sequence

__all__ = ["read_seq", "decompress_shape", "signature_ok"]

_DEFAULT_RASTERS = {"GradientRasterTime": 10e-6, "RadiofrequencyRasterTime": 1e-6, "AdcRasterTime": 1e-7,
                    "BlockDurationRaster": 10e-6}


def decompress_shape(packed, num_samples: int) -> np.ndarray:
    """Samples of a Pulseq shape: raw when all ``num_samples`` values are
    listed, else the run-length-encoded derivative integrated by cumsum."""
    packed = np.asarray(packed, dtype=np.float64)
    if packed.shape[0] == num_samples:
        return packed.copy()
    out: List[float] = []
    i, n = 0, packed.shape[0]
    while i < n:
        if i + 2 < n and packed[i] == packed[i + 1]:
            rep = packed[i + 2]
            if rep != int(rep) or rep < 0:
                raise ArgumentError("Malformed Pulseq shape: a repeat count must be a nonnegative integer.")
            out.extend([packed[i]] * (int(rep) + 2))
            i += 3
        else:
            out.append(packed[i])
            i += 1
    if len(out) != num_samples:
        raise ArgumentError(f"Pulseq shape decodes to {len(out)} samples, expected {num_samples}.")
    return np.cumsum(out)


def _sections(text: str) -> Dict[str, List[str]]:
    sections: Dict[str, List[str]] = {}
    current = None
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("[") and line.endswith("]"):
            current = line[1:-1].strip().upper()
            sections.setdefault(current, [])
            continue
        if current is None:
            raise ArgumentError("Pulseq file: content before the first section.")
        sections[current].append(line)
    return sections


def _numbers(line: str, n: int, what: str) -> List[float]:
    parts = line.split()
    if len(parts) != n:
        raise ArgumentError(f"Pulseq {what} line needs {n} fields: {line!r}")
    try:
        return [float(p) for p in parts]
    except ValueError:
        raise ArgumentError(f"Pulseq {what} line has a non-numeric field: {line!r}") from None


def _definitions(lines) -> Dict[str, object]:
    out: Dict[str, object] = {}
    for line in lines:
        key, *vals = line.split()
        try:
            nums = [float(v) for v in vals]
            out[key] = nums[0] if len(nums) == 1 else nums
        except ValueError:
            out[key] = " ".join(vals)
    return out


def _shapes(lines) -> Dict[int, np.ndarray]:
    shapes: Dict[int, np.ndarray] = {}
    i = 0
    while i < len(lines):
        head = lines[i].split()
        if len(head) != 2 or head[0] != "shape_id":
            raise ArgumentError(f"Pulseq [SHAPES]: expected 'shape_id N', got {lines[i]!r}")
        sid = int(head[1])
        cnt = lines[i + 1].split() if i + 1 < len(lines) else []
        if len(cnt) != 2 or cnt[0] != "num_samples":
            raise ArgumentError(f"Pulseq [SHAPES]: shape {sid} lacks num_samples.")
        num = int(cnt[1])
        j = i + 2
        vals = []
        while j < len(lines) and not lines[j].startswith("shape_id"):
            vals.append(float(lines[j]))
            j += 1
        shapes[sid] = decompress_shape(vals, num)
        i = j
    return shapes


def signature_ok(path: str) -> bool:
    """True when the file's ``[SIGNATURE]`` md5 matches its content (the text
    before the newline that precedes ``[SIGNATURE]``); False without one."""
    data = open(path, "rb").read()
    pos = data.find(b"\n[SIGNATURE]")
    if pos < 0:
        return False
    want = None
    for line in data[pos:].decode("ascii", "replace").splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0] == "Hash":
            want = parts[1].lower()
    return want is not None and hashlib.md5(data[:pos]).hexdigest() == want


def read_seq(path: str, gamma: float = GAMMA) -> Sequence:
    """Read a Pulseq 1.4 ``.seq`` file into a ``Sequence`` (``DEF`` holds the
    definitions, ``EXT`` the extension-list id of each block)."""
    with open(path, "r", encoding="utf-8", errors="replace") as f:
        sec = _sections(f.read())
    ver = sec.get("VERSION", [])
    version = {}
    for line in ver:
        k, v = line.split()[:2]
        version[k] = int(v)
    if (version.get("major"), version.get("minor")) != (1, 4):
        raise ArgumentError(f"Only Pulseq 1.4 files are supported (this file: {version.get('major')}."
                            f"{version.get('minor')}).")
    defs = _definitions(sec.get("DEFINITIONS", []))
    r = {k: float(defs.get(k, v)) for k, v in _DEFAULT_RASTERS.items()}
    shapes = _shapes(sec.get("SHAPES", []))

    def shape(sid, what):
        if sid not in shapes:
            raise ArgumentError(f"Pulseq {what} refers to missing shape {sid}.")
        return shapes[sid]

    grads: Dict[int, Grad] = {}
    for line in sec.get("TRAP", []):
        gid, amp, rise, flat, fall, delay = _numbers(line, 6, "[TRAP]")
        grads[int(gid)] = Grad(amp / gamma, flat / 1e6, rise / 1e6, fall / 1e6, delay / 1e6)
    for line in sec.get("GRADIENTS", []):
        gid, amp, amp_id, time_id, delay = _numbers(line, 5, "[GRADIENTS]")
        w = amp / gamma * shape(int(amp_id), "[GRADIENTS]")
        ras = r["GradientRasterTime"]
        if int(time_id) == 0:
            grads[int(gid)] = Grad(w, (w.shape[0] - 1) * ras, ras / 2, ras / 2, delay / 1e6)
        else:
            tt = shape(int(time_id), "[GRADIENTS]") * ras
            if tt.shape[0] != w.shape[0]:
                raise ArgumentError(f"Pulseq gradient {int(gid)}: time and amplitude shapes differ in length.")
            grads[int(gid)] = Grad(w, np.diff(tt), 0.0, 0.0, delay / 1e6 + tt[0], first=w[0], last=w[-1])
    rfs: Dict[int, RF] = {}
    for line in sec.get("RF", []):
        rid, amp, mag_id, ph_id, time_id, delay, freq, phase = _numbers(line, 8, "[RF]")
        mag = shape(int(mag_id), "[RF]")
        ph = shape(int(ph_id), "[RF]") if int(ph_id) else np.zeros_like(mag)
        if ph.shape[0] != mag.shape[0]:
            raise ArgumentError(f"Pulseq RF {int(rid)}: magnitude and phase shapes differ in length.")
        b1 = amp / gamma * mag * np.exp(1j * (2 * np.pi * ph + phase))
        ras = r["RadiofrequencyRasterTime"]
        if int(time_id) == 0:
            rfs[int(rid)] = RF(b1, (b1.shape[0] - 1) * ras, freq, delay / 1e6 + ras / 2)
        else:
            tt = shape(int(time_id), "[RF]") * ras
            if tt.shape[0] != b1.shape[0]:
                raise ArgumentError(f"Pulseq RF {int(rid)}: time and magnitude shapes differ in length.")
            rfs[int(rid)] = RF(b1, np.diff(tt), freq, delay / 1e6 + tt[0])
    adcs: Dict[int, ADC] = {}
    for line in sec.get("ADC", []):
        aid, num, dwell, delay, freq, phase = _numbers(line, 6, "[ADC]")
        dw = dwell / 1e9
        adcs[int(aid)] = ADC(int(num), (int(num) - 1) * dw, delay / 1e6 + dw / 2, freq, phase)

    blocks = [_numbers(line, 8, "[BLOCKS]") for line in sec.get("BLOCKS", [])]
    n = len(blocks)
    GR = np.empty((3, n), dtype=object)
    RFs = np.empty((1, n), dtype=object)
    ADCs = np.empty(n, dtype=object)
    DUR = np.zeros(n)
    EXT = np.zeros(n, dtype=np.int64)
    zero = Grad(0.0, 0.0)
    for j, (_, dur, rid, gx, gy, gz, aid, ext) in enumerate(blocks):
        for i, gid in enumerate((gx, gy, gz)):
            gid = int(gid)
            if gid and gid not in grads:
                raise ArgumentError(f"Pulseq block {j + 1} refers to missing gradient {gid}.")
            GR[i, j] = grads[gid] if gid else zero
        rid, aid = int(rid), int(aid)
        if rid and rid not in rfs:
            raise ArgumentError(f"Pulseq block {j + 1} refers to missing RF {rid}.")
        if aid and aid not in adcs:
            raise ArgumentError(f"Pulseq block {j + 1} refers to missing ADC {aid}.")
        RFs[0, j] = rfs[rid] if rid else RF(0.0, 0.0)
        ADCs[j] = adcs[aid] if aid else ADC(0, 0.0)
        events = max([g.dur for g in GR[:, j]] + [RFs[0, j].dur, ADCs[j].dur])
        DUR[j] = max(dur * r["BlockDurationRaster"], events) if math.isfinite(dur) else events
        EXT[j] = int(ext)
    seq = Sequence(GR, RFs, ADCs, DUR)
    seq.DEF = defs
    seq.EXT = EXT
    return seq

