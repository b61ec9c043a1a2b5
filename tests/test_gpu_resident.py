"""Device-resident phantoms (homs_resident_*): a simulation on a resident
phantom computes what homs_simulate computes on the same arrays, bit for bit,
whatever ran before it on the context and whatever runs beside it."""
import numpy as np
import pytest

import homs
from homs import workloads as W
from homs.model import BlochHighOrder, get_sim_ranges

pytestmark = pytest.mark.gpu


def _cases():
    obj, seq, st = W.high_order_workload(nspins=3000, nsteps=200, ncoils=32)
    obj2, seq2, _, _ = W.rf_acquisition_workload(3, 2, 11)
    parts2, exc2 = get_sim_ranges(seq2, 4, 5)
    return [(obj, seq, [(0, 200)], [False]), (obj2, seq2, parts2, exc2)]


@pytest.mark.parametrize("precision,mode", [("f64", "split"), ("f32", "split"), ("f64", "plain"), ("f32", "plain")])
def test_resident_equals_simulate(gpu_context, precision, mode):
    for obj, seq, parts, exc in _cases():
        if precision == "f32":
            obj, seq = obj.astype(np.float32), seq.astype(np.float32)
        params = {"sim_method": BlochHighOrder("1111"), "precision": precision, "homs_precision": mode}
        want = homs.simulate(obj, seq, sim_params=params, parts=parts, excitation=exc, context=gpu_context)
        with homs.ResidentPhantom(obj, precision, mode, context=gpu_context) as res:
            assert res.device_bytes() > 0
            for method in ("1111", "0110"):
                p = dict(params, sim_method=BlochHighOrder(method))
                got = homs.simulate(res, seq, sim_params=p, parts=parts, excitation=exc, context=gpu_context)
                ref = homs.simulate(obj, seq, sim_params=p, parts=parts, excitation=exc, context=gpu_context)
                assert got.dtype == ref.dtype
                assert np.array_equal(got, ref)
            again = homs.simulate(res, seq, sim_params=params, parts=parts, excitation=exc, context=gpu_context)
            assert np.array_equal(again, want)
        # The context's workspace was a view of the resident phantom: a plain
        # simulate afterwards must upload its own copy, not write through it.
        after = homs.simulate(obj, seq, sim_params=params, parts=parts, excitation=exc, context=gpu_context)
        assert np.array_equal(after, want)


def test_resident_shared_by_server_slots_and_sequences(gpu_context):
    obj, seq, _ = W.high_order_workload(nspins=20000, nsteps=500, ncoils=8)
    seqs = [seq]
    for k in range(3):  # the same phantom under other field waveforms
        s2 = W.high_order_workload(nspins=20000, nsteps=500, ncoils=8)[1]
        s2.h = s2.h * (1.0 + 0.1 * (k + 1))
        seqs.append(s2)
    params = {"sim_method": BlochHighOrder("1111"), "precision": "f64", "homs_precision": "split"}
    alone = [homs.simulate(obj, s, sim_params=params, parts=[(0, 500)], excitation=[False], context=gpu_context)
             for s in seqs]
    with homs.ResidentPhantom(obj, "f64", "split", context=gpu_context) as res:
        with homs.Server(slots=3) as srv:
            tickets = [(k, srv.submit(res, s, sim_params=params, parts=[(0, 500)], excitation=[False]))
                       for rep in range(3) for k, s in enumerate(seqs)]
            got = [(k, srv.result(t)) for k, t in tickets]
            spans = [srv.times(t) for _, t in tickets]
    for k, r in got:
        assert np.array_equal(r, alone[k])
    overlaps = sum(1 for i in range(len(spans)) for j in range(i + 1, len(spans))
                   if spans[i][1] < spans[j][2] and spans[j][1] < spans[i][2])
    assert overlaps > 0


def test_resident_mode_and_precision_must_match(gpu_context):
    obj, seq, _ = W.high_order_workload(nspins=100, nsteps=16, ncoils=2)
    with homs.ResidentPhantom(obj, "f64", "split", context=gpu_context) as res:
        with pytest.raises(homs.ArgumentError):
            homs.simulate(res, seq, sim_params={"homs_precision": "plain"}, parts=[(0, 16)], excitation=[False],
                          context=gpu_context)
        with pytest.raises(homs.ArgumentError):
            homs.simulate(res, seq, sim_params={"precision": "f32"}, parts=[(0, 16)], excitation=[False],
                          context=gpu_context)
    with pytest.raises(homs.ArgumentError):
        homs.simulate(res, seq, parts=[(0, 16)], excitation=[False], context=gpu_context)  # closed
