"""The reference's demo inputs as ``HO_Sequence``s: a Pulseq file plus measured
field dynamics from MATLAB files.

``demo3d_sequence`` follows demo3D/1_load_seq.jl:14-79 (a 3D stack-of-spirals
sequence whose readout blocks take field-camera gradients, interpolated onto
the gradient raster, with the nominal spoiler tail appended to the first
order rows and the partition rewinder before each readout replaced in h3;
Gx inverted; ADC phases negated for the RF phase compensation).
``demo2d_sequence`` follows demo2D/1_load_inputs.jl:22-52 (a 2D spiral whose
readout block takes the stitched field measurement, resampled to the ADC
times and differentiated to fields, with the nominal gradients copied into
h1..h3 of every block).  Both read MATLAB v5 files with ``scipy.io``.
"""
from __future__ import annotations

import copy

import numpy as np

from .model import GAMMA, ArgumentError
from .pulseq import read_seq
from .sequence import ADC, Grad, HO_Sequence, Sequence
from .trajectory import InterpTrajTime, traj2grad

__all__ = ["demo3d_sequence", "demo2d_sequence"]


def _loadmat(path):
    try:
        import scipy.io as sio
    except ImportError as e:  # pragma: no cover - scipy is part of the image
        raise ArgumentError("Reading MATLAB files needs scipy.") from e
    return sio.loadmat(path, squeeze_me=False, struct_as_record=True)


def _field(struct, name):
    return struct[name][0, 0]


def _negated_adc_phases(seq: Sequence) -> Sequence:
    """Copy of ``seq`` with every acquiring block's ADC phase negated (each
    block gets its own ADC object, so shared events are negated once per block)."""
    adcs = np.empty(len(seq), dtype=object)
    for j, a in enumerate(seq.ADC):
        if a.N > 0:
            a = copy.copy(a)
            a.phi = -a.phi
        adcs[j] = a
    return Sequence._raw(seq.GR, seq.RF, adcs, seq.DUR, seq.DEF, seq.EXT)


def demo3d_sequence(seq_path: str, params_path: str, skope_path: str, dtype=np.float32,
                    grad_raster: float = 10e-6, n_gz_pre: int = 34, n_spoiler: int = 300) -> HO_Sequence:
    """``hoseq`` of demo3D/1_load_seq.jl (Gx inverted, measured fields in the
    readout blocks, ADC phases negated).  ``dtype`` is the demo's ``T``."""
    seq = read_seq(seq_path)
    seq = Sequence._raw(seq.GR.copy(), seq.RF, seq.ADC, seq.DUR, seq.DEF, seq.EXT)
    seq.GR[0, :] = [-g for g in seq.GR[0, :]]  # invert Gx
    hoseq = HO_Sequence(seq)
    params = _loadmat(params_path)
    skope_p = params["skope"]
    dt_adc = float(np.asarray(_field(skope_p, "dt_adc")).reshape(-1)[0])
    n_sample_adc = int(np.asarray(_field(skope_p, "nSample_adc")).reshape(-1)[0])
    n_grad_adc = int(round(n_sample_adc * dt_adc / grad_raster))
    sk = _loadmat(skope_path)
    g_skope = (np.asarray(sk["g_skope"], dtype=np.float64) * 1e-3).astype(dtype)  # T/m
    t_g = np.asarray(sk["t_g"], dtype=dtype).reshape(-1)
    iadc = 0
    for j in range(len(seq)):
        if seq.GR[0, j].delay > 0 and seq.ADC[j].N > 0:
            if iadc >= g_skope.shape[0]:
                raise ArgumentError("The field-camera file has fewer readouts than the sequence.")
            g = InterpTrajTime(g_skope[iadc], grad_raster, -0.9 * grad_raster, t_g)
            n_delay = int(round(seq.GR[0, j].delay / grad_raster))
            for i in range(16):
                if i == 3:
                    prev = hoseq.GR_dfc[i, j - 1]
                    hoseq.GR_dfc[i, j - 1] = Grad(g[:n_gz_pre, i], (n_gz_pre - 1) * grad_raster, grad_raster / 2,
                                                  grad_raster / 2, prev.delay)
                amp = g[n_gz_pre + n_delay:, i]
                dur = (n_grad_adc - 1) * grad_raster
                if i in (1, 2):
                    dur = (n_grad_adc + n_spoiler - 1) * grad_raster
                    nominal = np.asarray(seq.GR[i - 1, j].A, dtype=np.float64).reshape(-1)
                    amp = np.concatenate([amp.astype(np.float64), nominal[-n_spoiler:]])
                hoseq.GR_dfc[i, j] = Grad(amp, dur, grad_raster / 2, grad_raster / 2, n_delay * grad_raster)
            iadc += 1
        else:
            for i in range(3):
                hoseq.GR_dfc[i + 1, j] = copy.copy(hoseq.SEQ.GR[i, j])
    out = HO_Sequence(_negated_adc_phases(seq), hoseq.GR_dfc)
    return out


def demo2d_sequence(seq_path: str, dfc_path: str, readout_block: int = 4) -> HO_Sequence:
    """``hoseqMeasured`` of demo2D/1_load_inputs.jl: blocks 3..end-3 of the
    file (1-based), nominal gradients in h1..h3, and the measured fields of
    the readout (0-based block ``readout_block`` of the kept blocks)."""
    d = _loadmat(dfc_path)

    def scalar(name):
        return float(np.asarray(d[name]).reshape(-1)[0])

    dt_measured, start, tau, dt_adc = scalar("dt_Measured"), scalar("startMeasured"), scalar("tauMeasured"), \
        scalar("dt_adc")
    kspha = np.asarray(d["ksphaMeasured"]).copy()
    kspha[:, 1] *= -1
    datatime = np.asarray(d["datatime"]).reshape(-1)
    n_sample = datatime.shape[0]
    # the measurement is single precision; the delay sum and the resampling follow it
    kspha = InterpTrajTime(kspha, np.float32(dt_measured), np.float32(start) + np.float32(tau) * np.float32(dt_adc),
                           datatime)
    bfield = traj2grad(kspha, np.float32(dt_adc), dim=1).astype(np.float64) / GAMMA * 1e3
    bfield = bfield.T * 1e-3
    full = read_seq(seq_path)
    seq = full[list(range(2, len(full) - 3))]
    t = dt_adc * (n_sample - 1)
    hoseq = HO_Sequence(seq)
    hoseq.GR_dfc[1:4, :] = hoseq.SEQ.GR
    for i in range(16):
        hoseq.GR_dfc[i, readout_block] = Grad(bfield[i], t, dt_adc / 2, dt_adc / 2, 0.0)
    return hoseq
