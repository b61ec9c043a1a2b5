"""Prepared plans replay a captured CUDA graph from their third run on; every
run computes the same signal, bit for bit, as the first (directly issued) run
and as homs_simulate."""
import numpy as np
import pytest

import homs
from homs import workloads as W
from homs.model import BlochHighOrder, get_sim_ranges

pytestmark = pytest.mark.gpu


def _check_plan(obj, seq, parts, exc, params, ctx):
    want = homs.simulate(obj, seq, sim_params=params, parts=parts, excitation=exc, context=ctx)
    with homs.prepare_simulation(obj, seq, sim_params=params, parts=parts, excitation=exc, context=ctx) as plan:
        assert plan.graph_state() == (0, "")
        runs = [plan.run() for _ in range(4)]
        state, why = plan.graph_state()
        assert state == 1, why
        states = [plan.run(return_type="state") for _ in range(2)]
    for r in runs:
        assert np.array_equal(r, want)
    assert np.array_equal(states[0].xy, states[1].xy) and np.array_equal(states[0].z, states[1].z)


@pytest.mark.parametrize("mode,precision", [("split", "f64"), ("split", "f32"), ("plain", "f64"), ("plain", "f32")])
def test_plan_graph_replays_equal_direct_runs(gpu_context, mode, precision):
    w = W.config(2, spins_stride=401)
    obj, seq = (w.obj, w.seq) if precision == "f64" else (w.obj.astype(np.float32), w.seq.astype(np.float32))
    params = {"sim_method": BlochHighOrder(w.mask), "precision": precision, "homs_precision": mode}
    _check_plan(obj, seq, w.parts, w.excitation, params, gpu_context)


def test_plan_graph_with_rf_blocks_and_tr_loop(gpu_context):
    obj, seq, _, _ = W.rf_acquisition_workload(3, 2, 11)
    parts, exc = get_sim_ranges(seq, 4, 5)
    for mode in ("split", "plain"):
        params = {"sim_method": BlochHighOrder("1111"), "precision": "f64", "homs_precision": mode}
        _check_plan(obj, seq, parts, exc, params, gpu_context)
    w = W.config(3, spins_stride=20011)  # 35 repetitions: RF, readout and fill segments
    params = {"sim_method": BlochHighOrder(w.mask), "precision": "f64", "homs_precision": "split"}
    _check_plan(w.obj, w.seq, w.parts, w.excitation, params, gpu_context)


def test_plan_graph_timing_is_recorded_on_replay(gpu_context):
    import ctypes
    from homs import _lib
    w = W.config(2, spins_stride=401)
    params = {"sim_method": BlochHighOrder(w.mask), "precision": "f64", "homs_precision": "split"}
    with homs.prepare_simulation(w.obj, w.seq, sim_params=params, parts=w.parts, excitation=w.excitation,
                                 context=gpu_context) as plan:
        for _ in range(3):
            plan.run()
        assert plan.graph_state()[0] == 1
        t = _lib.Timing()
        _lib.check(_lib.load().homs_plan_timing(plan.handle, ctypes.byref(t)))
    assert t.fused_launches == 4 and t.fused_kernel_ms > 0 and t.kernel_launches > t.fused_launches
