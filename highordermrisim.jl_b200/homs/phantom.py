"""Phantom builders on the GPU (homs_brain_phantom_*, homs_csm_birdcage).

``brain_phantom`` is hophantom_brain (src/phantom/hophantom_brain.jl:2-58) for a
volume of tissue classes that is already resampled to the target grid (what
load_phantom_mat returns; reading and resampling the reference's .mat files is
the caller's side).  ``csm_birdcage`` is csm_Birdcage
(src/phantom/csm/Birdcage.jl:21-42).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import Context
from .model import ArgumentError, DimensionMismatch, HO_Phantom

FIELD_STRENGTHS = {"1.5T": 0, "7T": 1}


def _ctx(context: Optional[Context]) -> Context:
    from . import _context
    return context or _context(0)


def brain_phantom(labels, target_res: Sequence[float], offcenter: Sequence[float] = (0.0, 0.0, 0.0), *,
                  fieldstrength: str = "1.5T", fieldmap=None, csm=None, name: Optional[str] = None,
                  context: Optional[Context] = None) -> HO_Phantom:
    """HO_Phantom of a brain class volume, built on the device.

    ``labels``: (nx, ny, nz) tissue classes (uint8) on the target grid;
    ``target_res``: voxel size in m; ``offcenter``: grid shift in m;
    ``fieldstrength``: "1.5T" or "7T" (SpinProperty's tables); ``fieldmap``:
    (nx, ny, nz) off-resonance in Hz, or None for the fat shift of
    b0_type = :fat; ``csm``: (nx, ny, nz, nc) complex receive map, or None for
    one unit coil.  Voxels with zero density are dropped; the rest keep
    column-major voxel order, as in the reference."""
    lab = np.asarray(labels)
    if lab.ndim != 3:
        raise DimensionMismatch("labels must be a 3D class volume (nx, ny, nz).")
    if lab.dtype != np.uint8:
        if lab.size and (lab.min() < 0 or lab.max() > 255 or not np.all(lab == np.round(lab))):
            raise ArgumentError("labels must hold tissue classes 0..255.")
        lab = lab.astype(np.uint8)
    if fieldstrength not in FIELD_STRENGTHS:
        raise ArgumentError("Field strength available: 1.5T, 7T")
    nx, ny, nz = lab.shape
    keep = []
    lab_f = np.asfortranarray(lab)
    keep.append(lab_f)
    spec = _lib.BrainSpec()
    spec.nx, spec.ny, spec.nz = nx, ny, nz
    spec.res[:] = [float(v) for v in target_res]
    spec.offcenter[:] = [float(v) for v in offcenter]
    spec.fieldstrength = FIELD_STRENGTHS[fieldstrength]
    spec.memory = _lib.HOMS_HOST
    spec.labels = lab_f.ctypes.data
    if fieldmap is not None:
        fm = np.asfortranarray(np.asarray(fieldmap, dtype=np.float64))
        if fm.shape != lab.shape:
            raise DimensionMismatch("fieldmap must have the shape of labels.")
        keep.append(fm)
        spec.fieldmap = fm.ctypes.data
    nc = 0
    if csm is not None:
        c = np.asfortranarray(np.asarray(csm, dtype=np.complex128))
        if c.ndim != 4 or c.shape[:3] != lab.shape:
            raise DimensionMismatch("csm must be (nx, ny, nz, ncoils).")
        keep.append(c)
        nc = c.shape[3]
        spec.csm = c.ctypes.data
    spec.ncoils = nc
    ctx = _ctx(context)
    lib = _lib.load()
    n = ctypes.c_int64()
    _lib.check(lib.homs_brain_phantom_count(ctx.handle, ctypes.byref(spec), ctypes.byref(n)), ctx.handle)
    ns = int(n.value)
    arrays = {k: np.zeros(ns) for k in ("x", "y", "z", "rho", "T1", "T2", "T2s", "dw")}
    csm_out = np.zeros((ns, max(nc, 1)), np.complex128, order="F")
    out = _lib.BrainOut()
    out.nspins = ns
    out.memory = _lib.HOMS_HOST
    for k, a in arrays.items():
        setattr(out, k, a.ctypes.data if ns else None)
    out.csm = csm_out.ctypes.data if ns else None
    if ns:
        _lib.check(lib.homs_brain_phantom_fill(ctx.handle, ctypes.byref(spec), ctypes.byref(out)), ctx.handle)
    return HO_Phantom(x=arrays["x"], y=arrays["y"], z=arrays["z"], rho=arrays["rho"], T1=arrays["T1"],
                      T2=arrays["T2"], T2s=arrays["T2s"], dw=arrays["dw"], csm=csm_out,
                      name=name or f"brain3D_{nx}x{ny}x{nz}_Cha{max(nc, 1)}")


def csm_birdcage(nx: int, ny: int, ncoils: int, relative_radius: float = 1.5,
                 context: Optional[Context] = None) -> np.ndarray:
    """(nx, ny, ncoils) complex birdcage receive map, computed on the device."""
    if nx < 1 or ny < 1 or ncoils < 1:
        raise ArgumentError("nX, nY and nCoil must be positive.")
    out = np.zeros((nx, ny, ncoils), np.complex128, order="F")
    ctx = _ctx(context)
    _lib.check(_lib.load().homs_csm_birdcage(ctx.handle, int(nx), int(ny), int(ncoils), float(relative_radius),
                                             out.ctypes.data, _lib.HOMS_HOST), ctx.handle)
    return out
