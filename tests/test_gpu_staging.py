"""Uploads from pageable host memory.

A pageable host input of 1 MiB or more is staged through the context's two
page-locked chunks (8 MiB each); a page-locked one is copied as it is.  The
same phantom, sequence and initial state are given once as pageable NumPy
arrays and once as page-locked copies: the results must agree bit for bit.
The phantom has an odd spin count (odd byte sizes) and its sensitivities
span three chunks.
"""
import ctypes

import numpy as np
import pytest

from homs import _lib
from homs import workloads as W
from homs.model import GAMMA, BlochHighOrder, count_block_adc

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t.numpy()


def _phantom(obj, dtype, pinned, keep):
    f = np.float64 if dtype == _lib.HOMS_F64 else np.float32
    c = np.complex128 if dtype == _lib.HOMS_F64 else np.complex64
    ns = len(obj.x)
    csm = np.asarray(obj.csm, dtype=c).reshape(ns, -1)
    cols = np.ascontiguousarray(csm.T)  # column-major csm: coil columns one after the other
    arrs = [np.ascontiguousarray(np.asarray(v, dtype=f)) for v in (obj.x, obj.y, obj.z, obj.rho, obj.T1, obj.T2, obj.dw)]
    if pinned:
        arrs = [_pinned(a) for a in arrs]
        cols = _pinned(cols)
    keep.extend(arrs + [cols])
    return _lib.Phantom(ns, csm.shape[1], dtype, _lib.HOMS_HOST, *[a.ctypes.data for a in arrs], cols.ctypes.data)


@pytest.mark.parametrize("mode,dtype", [("plain", _lib.HOMS_F64), ("split", _lib.HOMS_F32)])
def test_pageable_uploads_match_page_locked(gpu_context, mode, dtype):
    obj, seq, st = W.high_order_workload(nspins=600_001, nsteps=24, ncoils=2)
    lib = _lib.load()
    parts, exc = [(0, 12), (12, 24)], [False, False]
    cdt = np.complex128 if dtype == _lib.HOMS_F64 else np.complex64
    fdt = np.float64 if dtype == _lib.HOMS_F64 else np.float32
    nadc = int(sum(count_block_adc(seq.adc, parts)))
    out = []
    for pinned in (False, True):
        keep = []
        ph = _phantom(obj, dtype, pinned, keep)
        skeep = _lib._Keep()
        sq = _lib.host_sequence(seq, parts, exc, skeep, dtype, GAMMA)
        xy = np.ascontiguousarray(np.asarray(st.xy, dtype=cdt))
        z = np.ascontiguousarray(np.asarray(st.z, dtype=fdt))
        if pinned:
            xy, z = _pinned(xy), _pinned(z)
        else:
            xy, z = xy.copy(), z.copy()
        state = _lib.State(xy.ctypes.data, z.ctypes.data, _lib.HOMS_HOST)
        opts = _lib.RunOptions()
        opts.method = BlochHighOrder("1111").flags
        opts.mode = _lib.HOMS_SPLIT if mode == "split" else _lib.HOMS_PLAIN
        sig = np.zeros((max(nadc, 1), 2), dtype=cdt, order="F")
        _lib.check(lib.homs_simulate(gpu_context.handle, ctypes.byref(ph), ctypes.byref(sq), ctypes.byref(opts),
                                     ctypes.byref(state), ctypes.c_void_p(sig.ctypes.data), _lib.HOMS_HOST),
                   gpu_context.handle)
        out.append((sig.copy(), np.array(xy), np.array(z)))
    assert nadc > 0
    for a, b in zip(out[0], out[1]):
        assert a.dtype == b.dtype and a.shape == b.shape
        assert a.tobytes(order="F") == b.tobytes(order="F")
    assert np.abs(out[0][0]).max() > 0
