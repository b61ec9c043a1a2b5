"""The Python ctypes binding (homs/_lib.py) against the C header, on the CPU.

`_lib.load()` sets argtypes and restype on every entry point.  Each must
match its prototype in include/homs.h: the same number of arguments, each of
the same kind (pointer, 64- or 32-bit integer, double), and the same kind of
return value.  Loading the library needs no GPU."""
import ctypes

from homs import _lib

from test_julia_shim import header_functions


def _kind(t):
    if t is None:
        return None
    if t in (ctypes.c_void_p, ctypes.c_char_p) or (isinstance(t, type) and issubclass(t, ctypes._Pointer)):
        return "ptr"
    if t in (ctypes.c_int64, ctypes.c_longlong, ctypes.c_size_t, ctypes.c_uint64):
        return "i64"
    if t in (ctypes.c_int32, ctypes.c_int):
        return "i32"
    if t is ctypes.c_uint32:
        return "u32"
    if t is ctypes.c_double:
        return "f64"
    raise AssertionError(f"unexpected ctypes type {t}")


def test_every_header_function_is_bound_with_its_prototype():
    lib = _lib.load()
    hdr = header_functions()
    assert len(hdr) >= 30
    for name, (c_ret, c_args) in hdr.items():
        fn = getattr(lib, name)
        assert fn.argtypes is not None, f"{name} has no argtypes in homs/_lib.py"
        assert [_kind(a) for a in fn.argtypes] == c_args, (name, fn.argtypes, c_args)
        assert _kind(fn.restype) == c_ret, (name, fn.restype, c_ret)
