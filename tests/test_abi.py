"""libhoms loads and exports exactly the C ABI of include/homs.h (no GPU calls)."""
import ctypes
import os
import re

import pytest

from homs import _lib
from homs import workloads as W

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "homs.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(homs_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(homs_lib):
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(homs_lib, name), f"libhoms.so does not export {name}"
    assert sorted(_lib.EXPORTED) == sorted(n for n in names if n in _lib.EXPORTED)
    assert set(names) <= set(_lib.EXPORTED) | {n for n in names if hasattr(homs_lib, n)}


def test_abi_version_and_status_strings(homs_lib):
    assert homs_lib.homs_abi_version() == 1
    assert homs_lib.homs_status_string(0) == b"ok"
    assert homs_lib.homs_status_string(1) == b"invalid argument"
    assert homs_lib.homs_status_string(4) == b"timed out"


def test_count_adc_host_sequence(homs_lib):
    obj, seq, parts, exc = W.rf_acquisition_workload(3, 2, 11)
    keep = _lib._Keep()
    sq = _lib.host_sequence(seq, parts, exc, keep, _lib.HOMS_F64, 42.5774688e6)
    n = ctypes.c_int64(-1)
    assert homs_lib.homs_count_adc(ctypes.byref(sq), ctypes.byref(n)) == 0
    assert n.value == 16
    assert homs_lib.homs_count_adc(None, ctypes.byref(n)) == _lib.HOMS_EINVAL


def test_null_arguments_are_rejected_without_a_device(homs_lib):
    assert homs_lib.homs_context_create(0, None, None) == _lib.HOMS_EINVAL
    assert homs_lib.homs_simulate(None, None, None, None, None, None, 0) == _lib.HOMS_EINVAL
    assert homs_lib.homs_plan_destroy(None) == _lib.HOMS_EINVAL
    assert homs_lib.homs_last_error(None) == b"no context"


def test_context_without_gpu_fails_loudly(homs_lib):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = homs_lib.homs_context_create(0, None, ctypes.byref(h))
    assert st == _lib.HOMS_EUNSUPPORTED
    with pytest.raises(_lib.HomsError):
        _lib.Context(0)


def test_server_arguments_and_no_gpu(homs_lib):
    # Argument checks need no device; creation without a GPU fails loudly.
    assert homs_lib.homs_server_create(None, None) == _lib.HOMS_EINVAL
    assert homs_lib.homs_server_poll(None, 1) == _lib.HOMS_EINVAL
    assert homs_lib.homs_server_wait(None, 1, 1.0) == _lib.HOMS_EINVAL
    assert homs_lib.homs_server_destroy(None) == _lib.HOMS_EINVAL
    assert homs_lib.homs_server_error(None, 1) == b"no server"
    opts = _lib.ServerOptions()
    opts.slots = 100
    h = ctypes.c_void_p()
    assert homs_lib.homs_server_create(ctypes.byref(opts), ctypes.byref(h)) == _lib.HOMS_EINVAL
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        opts.slots = 2
        assert homs_lib.homs_server_create(ctypes.byref(opts), ctypes.byref(h)) == _lib.HOMS_EUNSUPPORTED
