"""Serving loop: continuous batching of mixed simulations.

Every result must be the same alone and in the mix (bit for bit: a request
runs the same kernels on the same inputs whatever runs beside it), requests
must overlap on the device when the budget allows, run one at a time when it
does not, and failures must come back on their own ticket.
"""
import numpy as np
import pytest

import homs
from conftest import nrmse
from homs import workloads as W
from homs.model import BlochHighOrder, get_sim_ranges

pytestmark = pytest.mark.gpu


def _requests():
    out = []
    obj, seq, st = W.high_order_workload(nspins=3000, nsteps=200, ncoils=32)
    out.append((obj, seq, [(0, 200)], [False], {"precision": "f64", "homs_precision": "split"}, "1111"))
    out.append((obj, seq, [(0, 200)], [False], {"precision": "f32"}, "1101"))
    obj2, seq2, st2 = W.high_order_workload(nspins=20000, nsteps=500, ncoils=8)
    out.append((obj2, seq2, [(0, 500)], [False], {"precision": "f64", "homs_precision": "split"}, "1110"))
    out.append((obj2, seq2, [(0, 500)], [False], {"precision": "f64"}, "0111"))
    obj3, seq3, _, _ = W.rf_acquisition_workload(3, 2, 11)
    parts3, exc3 = get_sim_ranges(seq3, 4, 5)
    out.append((obj3, seq3, parts3, exc3, {"precision": "f64", "homs_precision": "split"}, "1111"))
    w = W.config(1, spins_stride=7)
    out.append((w.obj, w.seq, w.parts, w.excitation, {"precision": "f64", "homs_precision": "split"}, w.mask))
    return out


def _params(extra, mask):
    return {"sim_method": BlochHighOrder(mask), **extra}


def test_alone_equals_in_mix(gpu_context):
    reqs = _requests()
    alone = [homs.simulate(o, s, sim_params=_params(p, m), parts=pa, excitation=ex, context=gpu_context)
             for o, s, pa, ex, p, m in reqs]
    with homs.Server(slots=3) as srv:
        # Every request twice, interleaved, so that copies run beside different neighbours.
        tickets = [(k, srv.submit(o, s, sim_params=_params(p, m), parts=pa, excitation=ex))
                   for rep in range(2) for k, (o, s, pa, ex, p, m) in enumerate(reqs)]
        got = [(k, srv.result(t)) for k, t in tickets]
        spans = [srv.times(t) for _, t in tickets]
    for k, r in got:
        assert r.shape == alone[k].shape
        assert np.array_equal(r, alone[k])
    for sub, start, fin in spans:
        assert sub <= start <= fin
    # With 3 slots and 12 requests some of them must have run at the same time.
    overlaps = sum(1 for i in range(len(spans)) for j in range(i + 1, len(spans))
                   if spans[i][1] < spans[j][2] and spans[j][1] < spans[i][2])
    assert overlaps > 0


def test_mixed_results_match_the_oracle(oracle, gpu_context):
    obj, seq, st = W.high_order_workload(nspins=777, nsteps=64, ncoils=8)
    method = BlochHighOrder("1111")
    ref = oracle.simulate_c(obj, seq, [(0, 64)], [False], method.flags)
    with homs.Server(slots=2) as srv:
        t1 = srv.submit(obj, seq, sim_params={"sim_method": method, "precision": "f64", "homs_precision": "split"},
                        parts=[(0, 64)], excitation=[False])
        t2 = srv.submit(obj, seq, sim_params={"sim_method": method, "precision": "f64"}, parts=[(0, 64)],
                        excitation=[False])
        split, plain = srv.result(t1)[:, :, 0], srv.result(t2)[:, :, 0]
    assert nrmse(split, ref[0]) <= 1e-6
    assert nrmse(plain, ref[0]) <= 1e-12


def test_budget_serialises_requests(gpu_context):
    reqs = [r for r in _requests() if r[4].get("homs_precision") == "split"]
    alone = [homs.simulate(o, s, sim_params=_params(p, m), parts=pa, excitation=ex, context=gpu_context)
             for o, s, pa, ex, p, m in reqs]
    # The server's own admission estimates of the split-mode requests.
    with homs.Server(slots=1) as probe:
        tickets = [probe.submit(o, s, sim_params=_params(p, m), parts=pa, excitation=ex) for o, s, pa, ex, p, m in reqs]
        est = [probe.estimate(t) for t in tickets]
        for t in tickets:
            probe.result(t)
    # Keep the requests (largest estimates first) for which a budget can admit
    # each one alone but no two together: one request in flight at a time.
    order = sorted(range(len(reqs)), key=lambda k: est[k])
    while len(order) > 2 and est[order[-1]] >= est[order[0]] + est[order[1]]:
        order.pop(0)
    reqs, alone = [reqs[k] for k in order], [alone[k] for k in order]
    e = sorted(est[k] for k in order)
    budget = (e[-1] + e[0] + e[1]) // 2
    assert e[-1] <= budget < e[0] + e[1]
    with homs.Server(slots=4, max_device_bytes=budget) as srv:
        tickets = [srv.submit(o, s, sim_params=_params(p, m), parts=pa, excitation=ex) for o, s, pa, ex, p, m in reqs]
        got = [srv.result(t) for t in tickets]
        spans = sorted(srv.times(t)[1:] for t in tickets)
    for r, a in zip(got, alone):
        assert np.array_equal(r, a)
    for (s0, f0), (s1, f1) in zip(spans, spans[1:]):
        assert s1 >= f0


def test_failures_stay_on_their_ticket(gpu_context):
    obj, seq, st = W.high_order_workload(nspins=100, nsteps=16, ncoils=2)
    with homs.Server(slots=2, max_device_bytes=64 << 20) as srv:
        # Larger than the whole admission budget.
        big = srv.submit(obj, seq, sim_params={"sim_method": BlochHighOrder("1111"), "precision": "f64",
                                               "homs_precision": "split"}, parts=[(0, 16)], excitation=[False])
        with pytest.raises(homs.HomsError) as e:
            srv.result(big)
        assert e.value.status == 2
    far, _, _ = W.high_order_workload(nspins=100, nsteps=16, ncoils=2)
    far.x[7] = 1000.0
    with homs.Server(slots=2) as srv:
        # A spin 1 km off-centre: its phase leaves the split path's fixed-point range.
        bad = srv.submit(far, seq, sim_params={"sim_method": BlochHighOrder("1111"), "precision": "f32",
                                               "homs_precision": "split"}, parts=[(0, 16)], excitation=[False])
        good = srv.submit(obj, seq, sim_params={"sim_method": BlochHighOrder("1111")}, parts=[(0, 16)],
                          excitation=[False])
        with pytest.raises(homs.HomsError) as e:
            srv.result(bad)
        assert e.value.status == 3
        assert srv.result(good).shape == (16, 2, 1)
        srv.release(good)
