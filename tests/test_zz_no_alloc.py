"""homs_coil_reduce_noalloc against homs_coil_reduce through the C ABI.

The allocation-free entry point keeps its split-K partials in a fixed device
array inside libhoms instead of context scratch.  It runs the same reduction
kernels, so its output must equal homs_coil_reduce's bit for bit, on two calls
in a row (the second must not see anything the first left in the array),
and after the first call on a device it allocates nothing: neither the
device's free memory nor the caller's own pooled allocator (torch here, as
CUDA.jl's would be for a Julia host) changes across further calls.
"""
import ctypes
import math

import numpy as np
import pytest

from homs import _lib

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 16 << 20
LD_PAD = 3


def _device(x, cdt):
    import torch
    return torch.as_tensor(np.asfortranarray(x), device="cuda:0").to(cdt).t().contiguous().t()


def _signal_buffer(nadc, nc, cdt):
    import torch
    # column-major (nadc + LD_PAD) x nc, canary-filled
    return torch.full((nc, nadc + LD_PAD), 7 - 3j, dtype=cdt, device="cuda:0")


def _args(dtype_code, states_t, csm_t, sig_t, ns, nadc, nc):
    return (dtype_code, ns, nadc, nc, ctypes.c_void_p(states_t.data_ptr()), max(ns, 1),
            ctypes.c_void_p(csm_t.data_ptr()), max(ns, 1), ctypes.c_void_p(sig_t.data_ptr()), nadc + LD_PAD)


def _problem(seed, ns, nadc, nc, precision):
    rng = np.random.default_rng(seed)
    states = rng.standard_normal((ns, nadc)) + 1j * rng.standard_normal((ns, nadc))
    csm = rng.standard_normal((ns, nc)) + 1j * rng.standard_normal((ns, nc))
    if precision == "f32":
        states = states.astype(np.complex64).astype(np.complex128)
        csm = csm.astype(np.complex64).astype(np.complex128)
    return states, csm


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_noalloc_matches_context_reduce_twice(gpu_context, precision):
    import torch
    lib = _lib.load()
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    code = _lib.HOMS_F64 if precision == "f64" else _lib.HOMS_F32
    stream = torch.cuda.Stream()
    # a larger problem first, then a smaller one that reuses part of the array
    for seed, (ns, nadc, nc) in enumerate([(9000, 40, 8), (1000, 13, 3)]):
        states, csm = _problem(100 + seed, ns, nadc, nc, precision)
        s_t, c_t = _device(states, cdt), _device(csm, cdt)
        want = _signal_buffer(nadc, nc, cdt)
        got = _signal_buffer(nadc, nc, cdt)
        torch.cuda.synchronize()
        _lib.check(lib.homs_coil_reduce(gpu_context.handle, *_args(code, s_t, c_t, want, ns, nadc, nc)),
                   gpu_context.handle)
        assert lib.homs_synchronize(gpu_context.handle) == 0
        st = ctypes.c_void_p(stream.cuda_stream)
        assert lib.homs_coil_reduce_noalloc(st, *_args(code, s_t, c_t, got, ns, nadc, nc)) == 0
        stream.synchronize()
        w, g = want.cpu().numpy(), got.cpu().numpy()
        assert np.array_equal(g, w)
        assert np.all(g[:, nadc:] == 7 - 3j)
        ref = states.T @ csm
        tol = 5e-6 if precision == "f32" else 5e-13
        scale = max(np.linalg.norm(ref), math.sqrt(ns * nadc * nc), 1)
        assert np.linalg.norm(g[:, :nadc].T - ref) / scale < tol


def test_noalloc_edges_and_limits(gpu_context):
    import torch
    lib = _lib.load()
    cdt = torch.complex128
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # no spins: signal columns are zeroed, padding untouched
    sig = _signal_buffer(5, 2, cdt)
    dummy = torch.zeros(1, dtype=cdt, device="cuda:0")
    assert lib.homs_coil_reduce_noalloc(st, *_args(_lib.HOMS_F64, dummy, dummy, sig, 0, 5, 2)) == 0
    torch.cuda.synchronize()
    s = sig.cpu().numpy()
    assert np.all(s[:, :5] == 0) and np.all(s[:, 5:] == 7 - 3j)
    # requests whose partials do not fit the fixed array are refused before any launch
    ns, nc = 256 * 65, 16
    nadc = SCRATCH_BYTES // (16 * 65 * nc) + 1
    assert 16 * 65 * nadc * nc > SCRATCH_BYTES
    big = _signal_buffer(nadc, nc, cdt)
    assert lib.homs_coil_reduce_noalloc(st, *_args(_lib.HOMS_F64, dummy, dummy, big, ns, nadc, nc)) == 1
    assert lib.homs_coil_reduce_noalloc(st, *_args(_lib.HOMS_F64, dummy, dummy, big, ns, nadc, 0)) == 1
    assert lib.homs_coil_reduce_noalloc(st, 7, 1, 1, 1, None, 1, None, 1, None, 1) == 1
    # the partials of the largest accepted f64 request exactly fill the array
    nadc_max = SCRATCH_BYTES // (16 * 65 * nc)
    states, csm = _problem(5, ns, nadc_max, nc, "f64")
    s_t, c_t = _device(states, cdt), _device(csm, cdt)
    got = _signal_buffer(nadc_max, nc, cdt)
    assert lib.homs_coil_reduce_noalloc(st, *_args(_lib.HOMS_F64, s_t, c_t, got, ns, nadc_max, nc)) == 0
    torch.cuda.synchronize()
    g = got.cpu().numpy()[:, :nadc_max].T
    ref = states.T @ csm
    assert np.linalg.norm(g - ref) / np.linalg.norm(ref) < 5e-13


def test_noalloc_allocates_nothing_after_set_up(gpu_context):
    import torch
    lib = _lib.load()
    cdt = torch.complex128
    stream = torch.cuda.Stream()
    st = ctypes.c_void_p(stream.cuda_stream)
    ns, nadc, nc = 4000, 24, 8
    states, csm = _problem(9, ns, nadc, nc, "f64")
    s_t, c_t = _device(states, cdt), _device(csm, cdt)
    out = [_signal_buffer(nadc, nc, cdt) for _ in range(3)]
    dummy = torch.zeros(1, dtype=cdt, device="cuda:0")
    # set-up: an empty request resolves the array on this device
    assert lib.homs_coil_reduce_noalloc(st, *_args(_lib.HOMS_F64, dummy, dummy, out[0], 0, 0, nc)) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    torch_alloc0 = torch.cuda.memory_allocated()
    torch_reserved0 = torch.cuda.memory_reserved()
    for k in range(3):
        assert lib.homs_coil_reduce_noalloc(st, *_args(_lib.HOMS_F64, s_t, c_t, out[k], ns, nadc, nc)) == 0
    stream.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == torch_alloc0
    assert torch.cuda.memory_reserved() == torch_reserved0
    first = out[0].cpu().numpy()
    for k in (1, 2):
        assert np.array_equal(out[k].cpu().numpy(), first)
