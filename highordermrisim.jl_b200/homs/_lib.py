"""ctypes binding of libhoms (include/homs.h).

The library is loaded from this package directory.  Nothing here falls back
to a CPU implementation: a missing or unloadable library raises
``HomsError`` and every failing C call raises with the library's message.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libhoms.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(PKG)), "include", "homs.h")

HOMS_OK, HOMS_EINVAL, HOMS_ENOMEM, HOMS_EUNSUPPORTED, HOMS_ETIMEDOUT, HOMS_ECUDA, HOMS_ECLOSED, HOMS_EBUSY = range(8)
HOMS_F32, HOMS_F64 = 0, 1
HOMS_HOST, HOMS_DEVICE = 0, 1
HOMS_PLAIN, HOMS_SPLIT = 0, 1

EXPORTED = [
    "homs_abi_version", "homs_status_string", "homs_context_create", "homs_context_destroy", "homs_last_error",
    "homs_synchronize", "homs_precession_block", "homs_excitation_block", "homs_coil_reduce", "homs_simulate",
    "homs_count_adc", "homs_plan_create", "homs_plan_run", "homs_plan_device_bytes", "homs_plan_timing",
    "homs_plan_destroy", "homs_coil_reduce_noalloc", "homs_server_create", "homs_server_submit", "homs_server_poll",
    "homs_server_wait", "homs_server_times", "homs_server_estimate", "homs_server_error", "homs_server_release",
    "homs_server_destroy",
    "homs_kspace", "homs_kspace_timing", "homs_resident_create", "homs_resident_device_bytes",
    "homs_resident_destroy", "homs_simulate_resident", "homs_server_submit_resident", "homs_plan_graph",
    "homs_brain_phantom_count", "homs_brain_phantom_fill", "homs_csm_birdcage", "homs_selftest_wait_timeout",
]


class HomsError(RuntimeError):
    """A libhoms call failed; ``status`` is the homs_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"libhoms status {status}: {message}")
        self.status = status


class Phantom(ctypes.Structure):
    _fields_ = [
        ("nspins", ctypes.c_int64), ("ncoils", ctypes.c_int32), ("dtype", ctypes.c_int), ("memory", ctypes.c_int),
        ("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p), ("rho", ctypes.c_void_p),
        ("T1", ctypes.c_void_p), ("T2", ctypes.c_void_p), ("dw", ctypes.c_void_p), ("csm", ctypes.c_void_p),
    ]


class Sequence(ctypes.Structure):
    _fields_ = [
        ("nnodes", ctypes.c_int64), ("dtype", ctypes.c_int), ("memory", ctypes.c_int),
        ("t", ctypes.c_void_p), ("dt", ctypes.c_void_p), ("gx", ctypes.c_void_p), ("gy", ctypes.c_void_p),
        ("gz", ctypes.c_void_p), ("b1", ctypes.c_void_p), ("df", ctypes.c_void_p), ("psi", ctypes.c_void_p),
        ("adc", ctypes.c_void_p), ("h", ctypes.c_void_p * 16), ("nblocks", ctypes.c_int32),
        ("block_first", ctypes.c_void_p), ("block_last", ctypes.c_void_p), ("block_excitation", ctypes.c_void_p),
        ("gamma", ctypes.c_double),
    ]


class RunOptions(ctypes.Structure):
    _fields_ = [("method", ctypes.c_uint32), ("mode", ctypes.c_int), ("reserved", ctypes.c_int32 * 6)]


class Timing(ctypes.Structure):
    _fields_ = [("fused_kernel_ms", ctypes.c_double), ("fused_launches", ctypes.c_int64),
                ("kernel_launches", ctypes.c_int64)]


class State(ctypes.Structure):
    _fields_ = [("xy", ctypes.c_void_p), ("z", ctypes.c_void_p), ("memory", ctypes.c_int)]


class BrainSpec(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64),
                ("res", ctypes.c_double * 3), ("offcenter", ctypes.c_double * 3), ("fieldstrength", ctypes.c_int32),
                ("ncoils", ctypes.c_int32), ("memory", ctypes.c_int), ("labels", ctypes.c_void_p),
                ("fieldmap", ctypes.c_void_p), ("csm", ctypes.c_void_p)]


class BrainOut(ctypes.Structure):
    _fields_ = [("nspins", ctypes.c_int64), ("memory", ctypes.c_int)] + [
        (name, ctypes.c_void_p) for name in ("x", "y", "z", "rho", "T1", "T2", "T2s", "dw", "csm")]


class ServerOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_int32), ("max_device_bytes", ctypes.c_int64),
                ("reserved", ctypes.c_int32 * 4)]


class RequestTimes(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_double), ("started", ctypes.c_double), ("finished", ctypes.c_double)]


_lib: Optional[ctypes.CDLL] = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libhoms.so (raises HomsError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise HomsError(HOMS_EUNSUPPORTED,
                        f"{path} is not built; run `python highordermrisim.jl_b200/homs/build.py`")
    lib = ctypes.CDLL(path)
    vp, i64, i32, u32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint32
    sig = {
        "homs_abi_version": (ctypes.c_int, []),
        "homs_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "homs_context_create": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(vp)]),
        "homs_context_destroy": (ctypes.c_int, [vp]),
        "homs_last_error": (ctypes.c_char_p, [vp]),
        "homs_synchronize": (ctypes.c_int, [vp]),
        "homs_precession_block": (ctypes.c_int, [vp, ctypes.POINTER(Phantom), ctypes.POINTER(Sequence), i64, i64, u32,
                                                 ctypes.POINTER(State), vp, i64]),
        "homs_excitation_block": (ctypes.c_int, [vp, ctypes.POINTER(Phantom), ctypes.POINTER(Sequence), i64, i64, u32,
                                                 ctypes.POINTER(State), vp, i64]),
        "homs_coil_reduce": (ctypes.c_int, [vp, ctypes.c_int, i64, i64, i32, vp, i64, vp, i64, vp, i64]),
        "homs_simulate": (ctypes.c_int, [vp, ctypes.POINTER(Phantom), ctypes.POINTER(Sequence),
                                         ctypes.POINTER(RunOptions), ctypes.POINTER(State), vp, ctypes.c_int]),
        "homs_count_adc": (ctypes.c_int, [ctypes.POINTER(Sequence), ctypes.POINTER(i64)]),
        "homs_plan_create": (ctypes.c_int, [vp, ctypes.POINTER(Phantom), ctypes.POINTER(Sequence),
                                            ctypes.POINTER(RunOptions), ctypes.POINTER(vp)]),
        "homs_plan_run": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.POINTER(State)]),
        "homs_plan_device_bytes": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_size_t)]),
        "homs_plan_timing": (ctypes.c_int, [vp, ctypes.POINTER(Timing)]),
        "homs_plan_destroy": (ctypes.c_int, [vp]),
        "homs_plan_graph": (ctypes.c_int, [vp, ctypes.POINTER(i32), ctypes.POINTER(ctypes.c_char_p)]),
        "homs_brain_phantom_count": (ctypes.c_int, [vp, ctypes.POINTER(BrainSpec), ctypes.POINTER(i64)]),
        "homs_brain_phantom_fill": (ctypes.c_int, [vp, ctypes.POINTER(BrainSpec), ctypes.POINTER(BrainOut)]),
        "homs_csm_birdcage": (ctypes.c_int, [vp, i64, i64, i32, ctypes.c_double, vp, ctypes.c_int]),
        "homs_selftest_wait_timeout": (ctypes.c_int, [vp, i64]),
        "homs_coil_reduce_noalloc": (ctypes.c_int, [vp, ctypes.c_int, i64, i64, i32, vp, i64, vp, i64, vp, i64]),
        "homs_server_create": (ctypes.c_int, [ctypes.POINTER(ServerOptions), ctypes.POINTER(vp)]),
        "homs_server_submit": (ctypes.c_int, [vp, ctypes.POINTER(Phantom), ctypes.POINTER(Sequence),
                                              ctypes.POINTER(RunOptions), ctypes.POINTER(State), vp, ctypes.c_int,
                                              ctypes.POINTER(i64)]),
        "homs_server_poll": (ctypes.c_int, [vp, i64]),
        "homs_server_wait": (ctypes.c_int, [vp, i64, ctypes.c_double]),
        "homs_server_times": (ctypes.c_int, [vp, i64, ctypes.POINTER(RequestTimes)]),
        "homs_server_estimate": (ctypes.c_int, [vp, i64, ctypes.POINTER(i64)]),
        "homs_server_error": (ctypes.c_char_p, [vp, i64]),
        "homs_server_release": (ctypes.c_int, [vp, i64]),
        "homs_server_destroy": (ctypes.c_int, [vp]),
        "homs_kspace": (ctypes.c_int, [vp, ctypes.POINTER(Sequence), i32, vp, vp, i64, vp, vp, vp, ctypes.c_int]),
        "homs_kspace_timing": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_double)]),
        "homs_resident_create": (ctypes.c_int, [vp, ctypes.POINTER(Phantom), ctypes.c_int, ctypes.POINTER(vp)]),
        "homs_resident_device_bytes": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_size_t)]),
        "homs_resident_destroy": (ctypes.c_int, [vp]),
        "homs_simulate_resident": (ctypes.c_int, [vp, vp, ctypes.POINTER(Sequence), ctypes.POINTER(RunOptions),
                                                  ctypes.POINTER(State), vp, ctypes.c_int]),
        "homs_server_submit_resident": (ctypes.c_int, [vp, vp, ctypes.POINTER(Sequence), ctypes.POINTER(RunOptions),
                                                       ctypes.POINTER(State), vp, ctypes.c_int,
                                                       ctypes.POINTER(i64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, ctx=None):
    if status != HOMS_OK:
        lib = load()
        msg = lib.homs_last_error(ctx).decode() if ctx else lib.homs_status_string(status).decode()
        raise HomsError(status, msg or lib.homs_status_string(status).decode())


class Context:
    """One device + one stream (``homs_context``)."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        lib = load()
        h = ctypes.c_void_p()
        st = lib.homs_context_create(int(device), ctypes.c_void_p(stream) if stream else None, ctypes.byref(h))
        if st != HOMS_OK:
            raise HomsError(st, f"homs_context_create(device={device}) failed: "
                                f"{lib.homs_status_string(st).decode()}")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            load().homs_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Keep:
    """Keeps numpy buffers alive while a C struct points into them."""

    def __init__(self):
        self.items = []

    def ptr(self, a: np.ndarray) -> int:
        self.items.append(a)
        return a.ctypes.data


def host_phantom(obj, keep: _Keep, dtype) -> Phantom:
    f = np.float64 if dtype == HOMS_F64 else np.float32
    c = np.complex128 if dtype == HOMS_F64 else np.complex64
    ns = len(obj.x)
    csm = np.asfortranarray(np.asarray(obj.csm, dtype=c).reshape(ns, -1))
    arr = lambda v: np.ascontiguousarray(np.asarray(v, dtype=f))  # noqa: E731
    return Phantom(ns, csm.shape[1], dtype, HOMS_HOST, keep.ptr(arr(obj.x)), keep.ptr(arr(obj.y)),
                   keep.ptr(arr(obj.z)), keep.ptr(arr(obj.rho)), keep.ptr(arr(obj.T1)), keep.ptr(arr(obj.T2)),
                   keep.ptr(arr(obj.dw)), keep.ptr(csm))


def host_sequence(seq, parts, excitation, keep: _Keep, dtype, gamma) -> Sequence:
    f = np.float64 if dtype == HOMS_F64 else np.float32
    c = np.complex128 if dtype == HOMS_F64 else np.complex64
    arr = lambda v: np.ascontiguousarray(np.asarray(v, dtype=f))  # noqa: E731
    nt = len(seq.t)
    h = np.ascontiguousarray(np.asarray(seq.h, dtype=f).reshape(16, nt))
    keep.items.append(h)
    hp = (ctypes.c_void_p * 16)(*[h[k].ctypes.data for k in range(16)])
    first = np.ascontiguousarray([p[0] for p in parts], dtype=np.int64)
    last = np.ascontiguousarray([p[1] for p in parts], dtype=np.int64)
    exc = np.ascontiguousarray(np.asarray(excitation, dtype=np.uint8))
    return Sequence(nt, dtype, HOMS_HOST, keep.ptr(arr(seq.t)), keep.ptr(arr(seq.dt)), keep.ptr(arr(seq.gx)),
                    keep.ptr(arr(seq.gy)), keep.ptr(arr(seq.gz)),
                    keep.ptr(np.ascontiguousarray(np.asarray(seq.b1, dtype=c))), keep.ptr(arr(seq.df)),
                    keep.ptr(arr(seq.psi)), keep.ptr(np.ascontiguousarray(np.asarray(seq.adc, dtype=np.uint8))),
                    hp, len(parts), keep.ptr(first), keep.ptr(last), keep.ptr(exc), float(gamma))
