"""Phantom builders on the GPU (homs_brain_phantom_*, homs_csm_birdcage).

``brain_phantom`` is hophantom_brain (src/phantom/hophantom_brain.jl:2-58) for a
volume of tissue classes that is already resampled to the target grid (what
load_phantom_mat returns).  ``hophantom_brain`` adds the host resampling of the
source volumes (class labels, receive map, off-resonance map) that the
reference does with Interpolations.jl before building.  ``csm_birdcage`` is
csm_Birdcage (src/phantom/csm/Birdcage.jl:21-42).
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


# --------------------------------------------------------------------------- resampling (host)
# The reference resamples its bundled volumes on the CPU with Interpolations.jl
# before building the phantom; these are restatements of those steps.

def _axis(n: int, res: float, location: float = 0.0) -> np.ndarray:
    """Voxel centres ((0:n-1) - (n-1)/2) * res + location."""
    return (np.arange(n) - (n - 1) / 2) * res + location


def _check_grid(target_res, target_matrix, location):
    if len(target_matrix) != 3 or not all(int(v) > 0 for v in target_matrix):
        raise ArgumentError("Target matrix dimensions must be positive.")
    if len(target_res) != 3 or not all(np.isfinite(v) and v > 0 for v in target_res):
        raise ArgumentError("Target voxel sizes must be finite and positive.")
    if len(location) != 3 or not all(np.isfinite(v) for v in location):
        raise ArgumentError("The sampling location must be finite.")


def _linear_axis(src: np.ndarray, coord: np.ndarray):
    """Lower index and weight of linear interpolation on the centres ``src``."""
    n = src.shape[0]
    if n == 1:
        return np.zeros(coord.shape[0], np.int64), np.zeros(coord.shape[0])
    step = src[1] - src[0]
    pos = (coord - src[0]) / step
    i0 = np.clip(np.floor(pos).astype(np.int64), 0, n - 2)
    return i0, pos - i0


def _trilinear(data: np.ndarray, axes_idx):
    """data[..., extra] sampled at the separable positions (i0, w) of each axis."""
    out = data
    for ax, (i0, w) in enumerate(axes_idx):
        lo = np.take(out, i0, axis=ax)
        hi = np.take(out, np.minimum(i0 + 1, out.shape[ax] - 1), axis=ax)
        shape = [1] * out.ndim
        shape[ax] = w.shape[0]
        w = w.reshape(shape)
        out = lo * (1 - w) + hi * w
    return out


def resample_labels(data, source_res, target_res, target_matrix, location=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Nearest-neighbour class volume on the target grid (load_phantom_mat,
    src/phantom/load_phantom_mat.jl:1-37): targets within the source's outer
    voxel faces take the nearest voxel (coordinates clamped to the outer
    centres, ties to even), targets beyond the faces are 0."""
    _check_grid(target_res, target_matrix, location)
    if len(source_res) != 3 or not all(np.isfinite(v) and v > 0 for v in source_res):
        raise ArgumentError("Source phantom voxel sizes must be finite and positive.")
    data = np.asarray(data)
    idx, valid = [], []
    for ax in range(3):
        n = data.shape[ax]
        src = _axis(n, source_res[ax])
        tgt = _axis(int(target_matrix[ax]), target_res[ax], location[ax])
        valid.append(np.abs(tgt) <= n * source_res[ax] / 2)
        c = np.clip(tgt, src[0], src[-1])
        pos = (c - src[0]) / source_res[ax] if n > 1 else np.zeros_like(c)
        idx.append(np.clip(np.rint(pos).astype(np.int64), 0, n - 1))
    out = data[np.ix_(*idx)].astype(np.uint8)
    mask = valid[0][:, None, None] & valid[1][None, :, None] & valid[2][None, None, :]
    return np.where(mask, out, np.uint8(0))


def resample_csm(data, source_res, target_res, target_matrix, location=(0.0, 0.0, 0.0)) -> np.ndarray:
    """(nx, ny, nz, nc) receive map on the target grid (_resample_csm,
    src/phantom/csm/Real_32cha.jl:62-95): trilinear on the source centres,
    coordinates clamped within the outer voxel faces, zero beyond them, and
    each nonzero receive vector normalised to unit summed squared magnitude."""
    _check_grid(target_res, target_matrix, location)
    data = np.asarray(data, dtype=np.complex128)
    if data.ndim != 4:
        raise DimensionMismatch("The receive map must be (nx, ny, nz, ncoils).")
    ai, valid = [], []
    for ax in range(3):
        n = data.shape[ax]
        src = _axis(n, source_res[ax])
        tgt = _axis(int(target_matrix[ax]), target_res[ax], location[ax])
        valid.append(np.abs(tgt) <= n * source_res[ax] / 2)
        ai.append(_linear_axis(src, np.clip(tgt, src[0], src[-1])))
    out = _trilinear(data, ai)
    mask = valid[0][:, None, None] & valid[1][None, :, None] & valid[2][None, None, :]
    out = out * mask[..., None]
    norm = np.sqrt(np.sum(np.abs(out) ** 2, axis=3, keepdims=True))
    return out / np.where(norm == 0, 1.0, norm)


def resample_b0(data, source_res, target_res, target_matrix, location=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Off-resonance map (Hz) on the target grid (b0_real,
    src/phantom/b0map/b0_real.jl:26-51): trilinear between the source
    centres, 0 outside them and where the source is NaN."""
    _check_grid(target_res, target_matrix, location)
    data = np.asarray(data, dtype=np.float64)
    ai, inside = [], []
    for ax in range(3):
        n = data.shape[ax]
        src = _axis(n, source_res[ax])
        tgt = _axis(int(target_matrix[ax]), target_res[ax], location[ax])
        inside.append((tgt >= src[0]) & (tgt <= src[-1]))
        ai.append(_linear_axis(src, np.clip(tgt, src[0], src[-1])))
    out = _trilinear(data, ai)
    mask = inside[0][:, None, None] & inside[1][None, :, None] & inside[2][None, None, :]
    out = np.where(mask, out, 0.0)
    out[np.isnan(out)] = 0.0
    return out


def hophantom_brain(brain, brain_res, target_res, target_matrix, location=(0.0, 0.0, 0.0),
                    offcenter=(0.0, 0.0, 0.0), *, fieldstrength: str = "1.5T", b0=None, b0_res=(4e-3,) * 3,
                    csm=None, csm_res=(4e-3,) * 3, ncoils: int = 32,
                    context: Optional[Context] = None) -> HO_Phantom:
    """hophantom_brain (src/phantom/hophantom_brain.jl:2-58) from source
    volumes: ``brain`` (class labels at ``brain_res``), ``b0`` (Hz at
    ``b0_res``; None for the fat shift of b0_type = :fat) and ``csm``
    (receive map at ``csm_res``, the first ``ncoils`` channels; None for one
    unit coil).  The volumes are resampled on the host as the reference does;
    the phantom is built on the device by ``brain_phantom``."""
    labels = resample_labels(brain, brain_res, target_res, target_matrix, location)
    fieldmap = None if b0 is None else resample_b0(b0, b0_res, target_res, target_matrix, location)
    cmap = None
    if csm is not None:
        c = np.asarray(csm)
        if not 1 <= ncoils <= c.shape[3]:
            raise ArgumentError(f"The receive map supports 1 to {c.shape[3]} coils.")
        cmap = resample_csm(c, csm_res, target_res, target_matrix, location)[..., :ncoils]
    return brain_phantom(labels, target_res, offcenter, fieldstrength=fieldstrength, fieldmap=fieldmap, csm=cmap,
                         context=context)


def generate_grid(fov, matrix_size) -> np.ndarray:
    """(nR, nP, nS, 3) voxel centres in metres (generate_grid,
    src/grid/Grid.jl:64-108): ((0:n-1) - (n-1)/2) * fov/n along each axis."""
    if len(fov) != 3 or len(matrix_size) != 3:
        raise ArgumentError("Both fov and matrix_size must be 3-element vectors.")
    if not all(np.isfinite(v) and v > 0 and float(v) == int(v) for v in matrix_size):
        raise ArgumentError("Matrix dimensions must be positive integers.")
    f = np.asarray(fov, dtype=np.float64)
    if not np.all(np.isfinite(f)) or np.any(f <= 0):
        raise ArgumentError("The field of view must be finite and positive.")
    n = [int(v) for v in matrix_size]
    grid = np.empty((n[0], n[1], n[2], 3))
    for k in range(3):
        shape = [1, 1, 1]
        shape[k] = n[k]
        grid[..., k] = _axis(n[k], f[k] / n[k]).reshape(shape)
    return grid


class Grid:
    """Voxel-centre grid of nX x nY x nZ voxels (Grid, src/grid/Grid.jl:1-58):
    ``x``, ``y``, ``z`` are flattened with x fastest, centred, in the
    spacing's float type; ``exchange_xy`` and ``reverse_x/y/z`` reorder them
    as the reference does."""

    def __init__(self, nX: int, nY: int, nZ: int, dx, dy, dz, exchange_xy=False, reverse_x=False, reverse_y=False,
                 reverse_z=False):
        if not all(int(n) == n and n > 0 for n in (nX, nY, nZ)):
            raise ArgumentError("Grid dimensions must be positive.")
        if not all(np.isfinite(v) and v > 0 for v in (dx, dy, dz)):
            raise ArgumentError("Grid spacing must be finite and positive.")
        dt = np.result_type(np.asarray(dx).dtype, np.asarray(dy).dtype, np.asarray(dz).dtype)
        if not np.issubdtype(dt, np.floating):
            dt = np.float64
        nX, nY, nZ = int(nX), int(nY), int(nZ)
        zz, yy, xx = np.meshgrid(np.arange(1, nZ + 1), np.arange(1, nY + 1), np.arange(1, nX + 1), indexing="ij")
        x = (xx.ravel() - (nX + 1) / 2) * float(dx)
        y = (yy.ravel() - (nY + 1) / 2) * float(dy)
        z = (zz.ravel() - (nZ + 1) / 2) * float(dz)
        if exchange_xy:
            x, y = y, x
        if reverse_x:
            x = x[::-1]
        if reverse_y:
            y = y[::-1]
        if reverse_z:
            z = z[::-1]
        self.nX, self.nY, self.nZ = nX, nY, nZ
        self.dx, self.dy, self.dz = dx, dy, dz
        self.x, self.y, self.z = (np.ascontiguousarray(v, dtype=dt) for v in (x, y, z))
        self.matrixSize = (nX, nY, nZ)
        self.resolution = (dx, dy, dz)

    def __repr__(self):
        r = [round(float(v) * 1e3, 2) for v in self.resolution]
        return f"Grid [ MatrixSize: {self.nX} x {self.nY} x {self.nZ}, Resolution: {r[0]} x {r[1]} x {r[2]} mm³ ]"
