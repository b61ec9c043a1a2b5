"""Failure detection without a GPU fault: a bounded device wait that nothing
completes runs out, the kernel records it in a device error word and
returns, and the host reports HOMS_ETIMEDOUT.  The same context then runs a
simulation correctly."""
import pytest

import homs
from conftest import nrmse
from homs import _lib
from homs import workloads as W
from homs.model import BlochHighOrder

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_the_context_stays_usable(oracle, gpu_context):
    lib = _lib.load()
    st = lib.homs_selftest_wait_timeout(gpu_context.handle, 2_000_000)  # ~1 ms at 2 GHz
    assert st == _lib.HOMS_ETIMEDOUT
    assert "timed out" in lib.homs_last_error(gpu_context.handle).decode()
    obj, seq, state = W.high_order_workload(nspins=500, nsteps=64, ncoils=4)
    method = BlochHighOrder("1111")
    ref = oracle.simulate_c(obj, seq, [(0, 64)], [False], method.flags, state.xy, state.z)
    got = homs.run_blocks(obj, seq, [(0, 64)], [False], method, "f64", "split", state, context=gpu_context)
    assert nrmse(got[0], ref[0]) <= 1e-6
    # twice in a row: the error word is cleared by every call
    assert lib.homs_selftest_wait_timeout(gpu_context.handle, 1_000) == _lib.HOMS_ETIMEDOUT


def test_selftest_rejects_budgets_out_of_range(gpu_context):
    lib = _lib.load()
    for budget in (0, 999, 5_000_000_000):
        assert lib.homs_selftest_wait_timeout(gpu_context.handle, budget) == _lib.HOMS_EINVAL
