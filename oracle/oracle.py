"""CPU oracle for the BlochHighOrder path.  TEST INFRASTRUCTURE ONLY.

Two independent restatements of HighOrderMRISim.jl's CPU Float64 path:

* ``simulate_c`` -- ctypes front end of ``homs_oracle.c`` (built by
  ``make -C oracle`` into ``oracle/_build/liboracle.so``), POSIX threads over spins.
* ``simulate_np`` -- a NumPy transcription of the Julia array code
  (``src/simulation/Bloch/BlochHighOrderSimulatitonMethod.jl:43-134`` and the
  block loop ``src/simulation/SimulatorCore.jl:96-152``), materialising
  Ns x Nt matrices exactly as the reference does.  For small cases only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module, and only as the checker.

Inputs are duck-typed: a phantom with ``x, y, z, rho, T1, T2, dw`` (float64,
length Ns) and ``csm`` (complex128, Ns x Nc); a sampled sequence with ``t, dt,
gx, gy, gz, b1, df, psi, adc, h`` (h is 16 x Nt); block ``parts`` as
0-based inclusive (first, last) node pairs and ``excitation`` flags per block.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

# KomaMRIBase's gyromagnetic ratio for 1H in Hz/T (the reference takes it
# from KomaMRIBase; its value is not defined inside the reference tree).
GAMMA = 42.5774688e6

HO0, HO1, HO2, HO3, DW_EXC, DW_PREC = 1, 2, 4, 8, 16, 32


class _Phantom(ctypes.Structure):
    _fields_ = [
        ("ns", ctypes.c_int64),
        ("nc", ctypes.c_int32),
        ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p),
        ("rho", ctypes.c_void_p), ("T1", ctypes.c_void_p), ("T2", ctypes.c_void_p),
        ("dw", ctypes.c_void_p), ("csm", ctypes.c_void_p),
    ]


class _Sequence(ctypes.Structure):
    _fields_ = [
        ("nt", ctypes.c_int64),
        ("t", ctypes.c_void_p), ("dt", ctypes.c_void_p),
        ("gx", ctypes.c_void_p), ("gy", ctypes.c_void_p), ("gz", ctypes.c_void_p),
        ("b1", ctypes.c_void_p), ("df", ctypes.c_void_p), ("psi", ctypes.c_void_p),
        ("adc", ctypes.c_void_p),
        ("h", ctypes.c_void_p * 16),
        ("nblocks", ctypes.c_int32),
        ("first", ctypes.c_void_p), ("last", ctypes.c_void_p), ("exc", ctypes.c_void_p),
        ("gamma", ctypes.c_double),
    ]


_lib = None


def build(force: bool = False) -> str:
    """Compile the C oracle (gcc, POSIX threads) into oracle/_build."""
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "homs_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        lib.oracle_simulate.restype = ctypes.c_int
        lib.oracle_simulate.argtypes = [
            ctypes.POINTER(_Phantom), ctypes.POINTER(_Sequence), ctypes.c_uint32,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
        ]
        lib.oracle_basis.restype = None
        lib.oracle_basis.argtypes = [ctypes.c_double] * 3 + [ctypes.c_void_p]
        lib.oracle_coil_combine.restype = None
        lib.oracle_coil_combine.argtypes = [
            ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ]
        _lib = lib
    return _lib


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def count_adc(adc, parts):
    """ADC samples owned by the blocks: ADC[first+1 .. last] (SimulatorCore.jl:115-116)."""
    adc = np.asarray(adc, dtype=bool)
    return int(sum(int(adc[f + 1:l + 1].sum()) for f, l in parts))


def simulate_c(phantom, seq, parts, excitation, method_flags, mxy0=None, mz0=None, nthreads=None,
               gamma=GAMMA):
    """Whole-sequence FP64 simulation by the C oracle.

    Returns (signal (Nadc x Nc complex128), mxy (Ns complex128), mz (Ns float64)).
    Initial state defaults to Mxy = 0, Mz = rho (BlochHighOrderSimulatitonMethod.jl:9-15).
    """
    lib = _load()
    keep = []

    def ptr(a):
        keep.append(a)
        return a.ctypes.data

    ns = len(phantom.x)
    csm = np.asfortranarray(np.asarray(phantom.csm, dtype=np.complex128).reshape(ns, -1))
    nc = csm.shape[1]
    ph = _Phantom(ns, nc, ptr(_f64(phantom.x)), ptr(_f64(phantom.y)), ptr(_f64(phantom.z)),
                  ptr(_f64(phantom.rho)), ptr(_f64(phantom.T1)), ptr(_f64(phantom.T2)),
                  ptr(_f64(phantom.dw)), ptr(csm))
    nt = len(seq.t)
    h = np.ascontiguousarray(np.asarray(seq.h, dtype=np.float64).reshape(16, nt))
    hptr = (ctypes.c_void_p * 16)(*[h[k].ctypes.data for k in range(16)])
    keep.append(h)
    first = np.ascontiguousarray([p[0] for p in parts], dtype=np.int64)
    last = np.ascontiguousarray([p[1] for p in parts], dtype=np.int64)
    exc = np.ascontiguousarray(np.asarray(excitation, dtype=np.uint8))
    b1 = np.ascontiguousarray(np.asarray(seq.b1, dtype=np.complex128))
    adc = np.ascontiguousarray(np.asarray(seq.adc, dtype=np.uint8))
    sq = _Sequence(nt, ptr(_f64(seq.t)), ptr(_f64(seq.dt)), ptr(_f64(seq.gx)), ptr(_f64(seq.gy)),
                   ptr(_f64(seq.gz)), ptr(b1), ptr(_f64(seq.df)), ptr(_f64(seq.psi)), ptr(adc), hptr,
                   len(parts), ptr(first), ptr(last), ptr(exc), float(gamma))
    nadc = count_adc(seq.adc, parts)
    mxy = np.zeros(ns, np.complex128) if mxy0 is None else np.array(mxy0, dtype=np.complex128)
    mz = _f64(phantom.rho).copy() if mz0 is None else np.array(mz0, dtype=np.float64)
    sig = np.zeros((nadc, nc), dtype=np.complex128, order="F")
    if nthreads is None:
        nthreads = max(1, min(len(os.sched_getaffinity(0)), 64))
    rc = lib.oracle_simulate(ctypes.byref(ph), ctypes.byref(sq), int(method_flags), mxy.ctypes.data,
                             mz.ctypes.data, sig.ctypes.data, nadc, int(nthreads))
    if rc != 0:
        raise ValueError(f"oracle_simulate failed with code {rc}")
    return np.asarray(sig), mxy, mz


def basis_c(x, y, z):
    out = np.zeros(16)
    _load().oracle_basis(float(x), float(y), float(z), out.ctypes.data)
    return out


def coil_combine_c(states, csm):
    """transpose(states)·csm in FP64 (states Ns x Nadc, csm Ns x Nc)."""
    states = np.asfortranarray(np.asarray(states, dtype=np.complex128))
    csm = np.asfortranarray(np.asarray(csm, dtype=np.complex128))
    ns, nadc = states.shape
    nc = csm.shape[1]
    sig = np.zeros((nadc, nc), np.complex128, order="F")
    _load().oracle_coil_combine(ns, nadc, nc, states.ctypes.data, csm.ctypes.data, sig.ctypes.data)
    return sig


# ---------------------------------------------------------------------------
# NumPy twin: a direct transcription of the Julia array code, block by block.
# ---------------------------------------------------------------------------

def basis_np(x, y, z):
    """Basis columns (Ns x 16), CPU expression order (BlochHighOrderSimulatitonMethod.jl:54-68)."""
    x2, y2, z2 = x * x, y * y, z * z
    r2 = (x2 + y2) + z2
    one = np.ones_like(x)
    return np.stack([
        one, x, y, z, x * y, z * y, 3.0 * z2 - r2, x * z, x2 - y2,
        (3.0 * y) * x2 - (y2 * y), (x * z) * y, (5.0 * z2 - r2) * y,
        5.0 * (z2 * z) - (3.0 * z) * r2, (5.0 * z2 - r2) * x, x2 * z - y2 * z, (x2 * x) - (3.0 * x) * y2,
    ], axis=1)


def _cmul(a, b):
    return (a.real * b.real - a.imag * b.imag) + 1j * (a.real * b.imag + a.imag * b.real)


def precession_np(phantom, seq, f, l, flags, mxy, mz, gamma=GAMMA):
    """run_spin_precession! for nodes f..l (BlochHighOrderSimulatitonMethod.jl:43-94).
    Updates mxy/mz in place and returns the block signal (Nadc_b x Nc)."""
    x, y, z = (np.asarray(v, np.float64)[:, None] for v in (phantom.x, phantom.y, phantom.z))
    h = np.asarray(seq.h, np.float64)[:, f:l + 1]
    g = [np.asarray(v, np.float64)[f:l + 1][None, :] for v in (seq.gx, seq.gy, seq.gz)]
    hr = [h[k][None, :] for k in range(16)]
    x2, y2, z2 = x * x, y * y, z * z
    r2 = (x2 + y2) + z2
    bzh = [None, x * hr[1], y * hr[2], z * hr[3], (x * y) * hr[4], (z * y) * hr[5], (3.0 * z2 - r2) * hr[6],
           (x * z) * hr[7], (x2 - y2) * hr[8], ((3.0 * y) * x2 - (y2 * y)) * hr[9], ((x * z) * y) * hr[10],
           ((5.0 * z2 - r2) * y) * hr[11], (5.0 * (z2 * z) - (3.0 * z) * r2) * hr[12],
           ((5.0 * z2 - r2) * x) * hr[13], (x2 * z - y2 * z) * hr[14], ((x2 * x) - (3.0 * x) * y2) * hr[15]]
    bz0 = hr[0] if flags & HO0 else 0.0
    bz1 = (bzh[1] + bzh[2]) + bzh[3] if flags & HO1 else (x * g[0] + y * g[1]) + z * g[2]
    bz2 = (((bzh[4] + bzh[5]) + bzh[6]) + bzh[7]) + bzh[8] if flags & HO2 else 0.0
    bz3 = (((((bzh[9] + bzh[10]) + bzh[11]) + bzh[12]) + bzh[13]) + bzh[14]) + bzh[15] if flags & HO3 else 0.0
    bz = ((bz0 + bz1) + bz2) + bz3
    if flags & DW_PREC:
        bz = bz + np.asarray(phantom.dw, np.float64)[:, None] / (2.0 * np.pi * gamma)
    bz = np.broadcast_to(bz, (len(phantom.x), l - f + 1))
    dt = np.asarray(seq.dt, np.float64)[f:l]
    y_ = (bz[:, 1:] + bz[:, :-1]) * dt[None, :]
    phi = (-(2.0 * np.pi * gamma)) * (0.5 * np.cumsum(y_, axis=1))
    tp = np.cumsum(dt)
    T2 = np.asarray(phantom.T2, np.float64)[:, None]
    e = np.exp(0.0 - tp[None, :] / T2)
    ez = e * np.cos(phi) + 1j * (e * np.sin(phi))
    m0 = mxy[:, None].copy()
    states = _cmul(np.broadcast_to(m0, ez.shape), ez)
    if l > f:
        mxy[:] = states[:, -1]
    dur = tp[-1] if len(tp) else 0.0
    e1 = np.exp(-dur / np.asarray(phantom.T1, np.float64))
    mz[:] = mz * e1 + np.asarray(phantom.rho, np.float64) * (1.0 - e1)
    adc = np.asarray(seq.adc, bool)[f + 1:l + 1]
    sel = states[:, adc]
    csm = np.asarray(phantom.csm, np.complex128).reshape(len(phantom.x), -1)
    return sel.T @ csm


def excitation_np(phantom, seq, f, l, flags, mxy, mz, gamma=GAMMA):
    """run_spin_excitation! for nodes f..l (BlochHighOrderSimulatitonMethod.jl:100-134)."""
    twopig = 2.0 * np.pi * gamma
    x, y, z = (np.asarray(v, np.float64) for v in (phantom.x, phantom.y, phantom.z))
    rho, T1, T2 = (np.asarray(v, np.float64) for v in (phantom.rho, phantom.T1, phantom.T2))
    csm = np.asarray(phantom.csm, np.complex128).reshape(len(x), -1)
    psi = np.asarray(seq.psi, np.float64)
    mxy[:] = _cmul(mxy, np.cos(-psi[f]) + 1j * np.sin(-psi[f]))
    off = np.asarray(phantom.dw, np.float64) / twopig if flags & DW_EXC else 0.0
    out = []
    for n in range(f, l):
        dbz = off - seq.df[n] / gamma
        bz = ((seq.gx[n] * x + seq.gy[n] * y) + seq.gz[n] * z) + dbz
        b1 = complex(seq.b1[n])
        B = np.sqrt(np.hypot(b1.real, b1.imag) ** 2 + bz * bz)
        B = np.where(B == 0.0, np.finfo(np.float64).eps, B)
        phi = -twopig * (B * seq.dt[n])
        sh, ch = np.sin(phi / 2.0), np.cos(phi / 2.0)
        nz = bz / B
        nx = (b1.real / B) + 1j * (b1.imag / B)
        alpha = ch + 1j * (-(nz * sh))
        beta = (nx.imag * sh) + 1j * (-(nx.real * sh))
        ca = np.conj(alpha)
        t1 = _cmul(2.0 * ca.real + 1j * (2.0 * ca.imag), beta) * mz
        t2 = _cmul(_cmul(ca, ca), mxy)
        t3 = _cmul(_cmul(beta, beta), np.conj(mxy))
        nxy = (t1 + t2) - t3
        nzz = (np.abs(alpha) ** 2 - np.abs(beta) ** 2) * mz - 2.0 * _cmul(_cmul(alpha, beta), np.conj(mxy)).real
        mxy[:] = nxy * np.exp(-seq.dt[n] / T2)
        e1 = np.exp(-seq.dt[n] / T1)
        mz[:] = nzz * e1 + rho * (1.0 - e1)
        if seq.adc[n + 1]:
            s = _cmul(mxy, np.cos(psi[n + 1]) + 1j * np.sin(psi[n + 1]))
            out.append(s @ csm)
    mxy[:] = _cmul(mxy, np.cos(psi[l]) + 1j * np.sin(psi[l]))
    if out:
        return np.stack(out, axis=0)
    return np.zeros((0, csm.shape[1]), np.complex128)


def simulate_np(phantom, seq, parts, excitation, method_flags, mxy0=None, mz0=None, gamma=GAMMA):
    """run_sim_time_iter! over blocks with the NumPy twin (single spin part)."""
    ns = len(phantom.x)
    mxy = np.zeros(ns, np.complex128) if mxy0 is None else np.array(mxy0, dtype=np.complex128)
    mz = np.array(phantom.rho, dtype=np.float64) if mz0 is None else np.array(mz0, dtype=np.float64)
    blocks = []
    for (f, l), ex in zip(parts, excitation):
        if ex:
            blocks.append(excitation_np(phantom, seq, f, l, method_flags, mxy, mz, gamma))
        else:
            blocks.append(precession_np(phantom, seq, f, l, method_flags, mxy, mz, gamma))
    nc = np.asarray(phantom.csm).reshape(ns, -1).shape[1]
    sig = np.concatenate(blocks, axis=0) if blocks else np.zeros((0, nc), np.complex128)
    return sig, mxy, mz


# ---------------------------------------------------------------------------
# Encoding export: grad2kspace (src/datatypes/HO_Sequence.jl:257-287).
# ---------------------------------------------------------------------------

def cumtrapz_np(dt, x):
    """KomaMRICore's cumtrapz for vectors: cumsum((x[2:end] + x[1:end-1]) .* (dt / 2))
    (third-party, KomaMRICore 0.14.0; used at HO_Sequence.jl:268)."""
    x = np.asarray(x, dtype=np.float64)
    return np.cumsum((x[1:] + x[:-1]) * (np.asarray(dt, dtype=np.float64) / 2))


def kfoldperm_parts(n, breaks):
    """Parts of 1:n cut at 1-based ``breaks``, as KomaMRIBase's
    kfoldperm(n, 1; breaks) builds them (HO_Sequence.jl:264): each break
    starts a new part; returned 0-based as (first, last_exclusive)."""
    b = sorted(set([1, n + 1] + [int(v) for v in breaks]))
    return [(b[i] - 1, b[i + 1] - 1) for i in range(len(b) - 1)]


def grad2kspace_np(seq, rf_start, rf_sign, gamma=GAMMA, q_times=None):
    """k-space of the 19 columns gx, gy, gz, h0..h15 of a sampled sequence
    (grad2kspace, HO_Sequence.jl:261-287), part by part exactly as the loop at
    :266-278, with the RF breaks given as 0-based interval indices
    ``rf_start`` and their signs (0 excitation, -1 refocusing, +1 other or
    skipped; :272-274).  Returns (k (m x 19), k at ``q_times`` (nq x 19)),
    the latter by linear interpolation over the knots t[n] + dt[n] with 0
    outside them (:279-286)."""
    t = np.asarray(seq.t, dtype=np.float64)
    dt = np.asarray(seq.dt, dtype=np.float64)
    m = t.shape[0] - 1
    cols = [seq.gx, seq.gy, seq.gz] + [seq.h[i] for i in range(16)]
    parts = kfoldperm_parts(m, [s + 1 for s in rf_start])
    k = np.zeros((m, len(cols)))
    for term, g in enumerate(cols):
        g = np.asarray(g, dtype=np.float64)
        previous = 0.0
        for r, (a, b) in enumerate(parts):
            k[a:b, term] = cumtrapz_np(dt[a:b], g[a:b + 1])
            if r > 0:
                k[a:b, term] += rf_sign[r - 1] * previous
            previous = k[b - 1, term]
    kspace = gamma * k
    if q_times is None:
        return kspace, np.zeros((0, len(cols)))
    knots = t[:-1] + dt
    q = np.asarray(q_times, dtype=np.float64)
    kq = np.zeros((q.shape[0], len(cols)))
    for j, tau in enumerate(q):
        if tau < knots[0] or tau > knots[-1]:
            continue
        n = int(np.searchsorted(knots, tau, side="right")) - 1
        if n == m - 1:
            kq[j] = kspace[n]
        else:
            w = (tau - knots[n]) / (knots[n + 1] - knots[n])
            kq[j] = kspace[n] + w * (kspace[n + 1] - kspace[n])
    return kspace, kq


# ---------------------------------------------------------------------------
# Phantom builders: hophantom_brain (src/phantom/hophantom_brain.jl:2-58),
# SpinProperty (src/phantom/SpinProperty.jl:1-118), generate_grid
# (src/grid/Grid.jl:78-108), csm_Birdcage (src/phantom/csm/Birdcage.jl:21-42).
# ---------------------------------------------------------------------------

# class: (rho, T1 ms, T2 ms, T2s ms) at 1.5 T (SpinProperty.jl:12-59) and 7 T (:62-118)
_TISSUE_1P5T = {23: (1, 2569, 329, 58), 46: (.86, 833, 83, 69), 70: (.77, 500, 70, 61), 93: (1, 350, 70, 58),
                116: (1, 900, 47, 30), 139: (.7, 569, 329, 58), 162: (0, 0, 0, 0), 185: (0, 0, 0, 0),
                209: (.77, 500, 70, 61), 232: (1, 2569, 329, 58), 255: (.77, 500, 70, 61)}
_TISSUE_7T = {23: (1, 4400, 329, 58), 46: (.86, 2100, 50, 33), 70: (.77, 1200, 40, 27), 93: (1, 580, 46, 25),
              116: (1, 1700, 30, 23), 139: (.7, 1700, 30, 23), 162: (0, 0, 0, 0), 185: (0, 0, 0, 0),
              209: (.77, 1200, 40, 27), 232: (1, 4400, 329, 58), 255: (.77, 1200, 40, 27)}


def spin_property_np(labels, fieldstrength="1.5T"):
    """T1, T2, T2s (s) and rho per voxel: the class tables times 1e-3."""
    table = {"1.5T": _TISSUE_1P5T, "7T": _TISSUE_7T}[fieldstrength]
    lab = np.asarray(labels)
    rho, t1, t2, t2s = (np.zeros(lab.shape) for _ in range(4))
    for c, (r, a, b, d) in table.items():
        sel = lab == c
        rho[sel], t1[sel], t2[sel], t2s[sel] = float(r), float(a), float(b), float(d)
    return t1 * 1e-3, t2 * 1e-3, t2s * 1e-3, rho


def generate_grid_np(fov, matrix_size):
    """Voxel centres (n1, n2, n3, 3): ((0:n-1) - (n-1)/2) * fov/n per axis."""
    fov = np.asarray(fov, dtype=np.float64)
    n = [int(v) for v in matrix_size]
    spacing = fov / np.asarray(n, dtype=np.float64)
    axes = [(np.arange(n[k], dtype=np.float64) - (n[k] - 1) / 2) * spacing[k] for k in range(3)]
    grid = np.empty((n[0], n[1], n[2], 3))
    grid[..., 0] = axes[0][:, None, None]
    grid[..., 1] = axes[1][None, :, None]
    grid[..., 2] = axes[2][None, None, :]
    return grid


def brain_phantom_np(labels, target_res, offcenter=(0.0, 0.0, 0.0), fieldstrength="1.5T", fieldmap=None, csm=None):
    """Spin arrays of hophantom_brain for a resampled class volume: dict of
    x, y, z, rho, T1, T2, T2s, dw (Ns) and csm (Ns x Nc, Nc = 1 unit coil
    when csm is None), voxels with rho != 0 in column-major order."""
    lab = np.asarray(labels)
    matrix = lab.shape
    fov = np.asarray(matrix, dtype=np.float64) * np.asarray(target_res, dtype=np.float64)
    xyz = generate_grid_np(fov, matrix)
    x = xyz[..., 0] + offcenter[0]
    y = xyz[..., 1] + offcenter[1]
    z = xyz[..., 2] + offcenter[2]
    t1, t2, t2s, rho = spin_property_np(lab, fieldstrength)
    if fieldmap is None:
        dw_fat = -220 * (2 * np.pi)
        dw = np.where((lab == 93) | (lab == 209), dw_fat, -0.0)
    else:
        dw = np.asarray(fieldmap, dtype=np.float64) * (2 * np.pi)
    keep = (rho != 0).ravel(order="F")
    f = lambda a: np.asarray(a).ravel(order="F")[keep]  # noqa: E731
    out = {"x": f(x), "y": f(y), "z": f(z), "rho": f(rho), "T1": f(t1), "T2": f(t2), "T2s": f(t2s), "dw": f(dw)}
    if csm is None:
        out["csm"] = np.ones((int(keep.sum()), 1), np.complex128)
    else:
        c = np.asarray(csm, dtype=np.complex128)
        out["csm"] = c.reshape(-1, c.shape[-1], order="F")[keep]
    return out


def csm_birdcage_np(nx, ny, ncoils, relative_radius=1.5):
    """csm_Birdcage: (nx, ny, ncoils) complex, 1/r cis(phi) per coil, RSS-normalised."""
    out = np.zeros((nx, ny, ncoils), np.complex128)
    xs = np.arange(nx, dtype=np.float64)[:, None]
    ys = np.arange(ny, dtype=np.float64)[None, :]
    for c in range(ncoils):
        ang = c * (2 * np.pi / ncoils)
        coilx = relative_radius * np.cos(ang)
        coily = relative_radius * np.sin(ang)
        y_co = (ys - ny / 2) / (ny / 2) - coily
        x_co = (xs - nx / 2) / (nx / 2) - coilx
        rr = np.sqrt(x_co * x_co + y_co * y_co)
        phi = np.arctan2(x_co, -y_co) + (-ang)
        out[:, :, c] = (1 / rr) * (np.cos(phi) + 1j * np.sin(phi))
    norm = np.sqrt(np.sum(np.abs(out) ** 2, axis=2, keepdims=True))
    return out / norm
