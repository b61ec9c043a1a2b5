"""Split-precision tcgen05 path vs the FP64 CPU oracle (signal NRMSE <= 1e-6)."""
import numpy as np
import pytest

import homs
from conftest import nrmse
from homs import workloads as W
from homs.model import BlochHighOrder, get_sim_ranges

pytestmark = pytest.mark.gpu

SPLIT_NRMSE = 1e-6


def oracle_run(o, obj, seq, parts, exc, method, state=None):
    return o.simulate_c(obj, seq, parts, exc, method.flags, None if state is None else state.xy,
                        None if state is None else state.z)


def split_run(obj, seq, parts, exc, method, state=None):
    return homs.run_blocks(obj, seq, parts, exc, method, "f64", "split", state)


@pytest.mark.parametrize("mask", [format(m, "04b") for m in range(16)])
@pytest.mark.parametrize("ncoils", [1, 3, 32])
def test_split_fixture_all_masks(oracle, gpu_context, mask, ncoils):
    obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=ncoils)
    method = BlochHighOrder(mask)
    ref = oracle_run(oracle, obj, seq, [(0, 32)], [False], method, st)
    got = split_run(obj, seq, [(0, 32)], [False], method, st)
    assert nrmse(got[0], ref[0]) <= SPLIT_NRMSE
    assert nrmse(got[1], ref[1]) <= 1e-12
    assert nrmse(got[2], ref[2]) <= 1e-12


@pytest.mark.parametrize("nspins", [1, 31, 32, 33, 255, 257, 4099])
@pytest.mark.parametrize("nsteps", [1, 127, 128, 129, 300])
def test_split_tails(oracle, gpu_context, nspins, nsteps):
    obj, seq, st = W.high_order_workload(nspins=nspins, nsteps=nsteps, ncoils=8)
    method = BlochHighOrder("1111")
    ref = oracle_run(oracle, obj, seq, [(0, nsteps)], [False], method, st)
    got = split_run(obj, seq, [(0, nsteps)], [False], method, st)
    assert nrmse(got[0], ref[0]) <= SPLIT_NRMSE


@pytest.mark.parametrize("scenario", [(0, 0, 11, True), (3, 2, 11, True), (5, 2, 0, True)])
def test_split_with_rf_blocks(oracle, gpu_context, scenario):
    obj, seq, _, _ = W.rf_acquisition_workload(*scenario)
    parts, exc = get_sim_ranges(seq, 4, 5)
    method = BlochHighOrder("1111")
    ref = oracle_run(oracle, obj, seq, parts, exc, method)
    got = split_run(obj, seq, parts, exc, method)
    assert nrmse(got[0], ref[0]) <= SPLIT_NRMSE
    assert nrmse(got[1], ref[1]) <= 1e-10


def test_split_config0_full(oracle, gpu_context):
    w = W.config(0)
    method = BlochHighOrder(w.mask)
    ref = oracle_run(oracle, w.obj, w.seq, w.parts, w.excitation, method)
    got = split_run(w.obj, w.seq, w.parts, w.excitation, method)
    assert nrmse(got[0], ref[0]) <= SPLIT_NRMSE


@pytest.mark.parametrize("cfg,stride", [(1, 41), (2, 401), (2, 97), (3, 2003)])
def test_split_config_subsample(oracle, gpu_context, cfg, stride):
    w = W.config(cfg, spins_stride=stride)
    assert np.count_nonzero(w.obj.rho) > len(w.obj) // 4
    method = BlochHighOrder(w.mask)
    ref = oracle_run(oracle, w.obj, w.seq, w.parts, w.excitation, method)
    assert np.linalg.norm(ref[0]) > 0
    got = split_run(w.obj, w.seq, w.parts, w.excitation, method)
    assert nrmse(got[0], ref[0]) <= SPLIT_NRMSE
    # The state leaves the split path through the FP64 segment-end update.
    assert nrmse(got[1], ref[1]) <= 1e-10


def test_split_more_coils_than_one_group(oracle, gpu_context):
    # 40 coils run as two coil groups (32 + 8) of the tcgen05 kernel.
    obj, seq, st = W.high_order_workload(nspins=700, nsteps=64, ncoils=40)
    method = BlochHighOrder("1111")
    ref = oracle_run(oracle, obj, seq, [(0, 64)], [False], method, st)
    got = split_run(obj, seq, [(0, 64)], [False], method, st)
    assert nrmse(got[0], ref[0]) <= SPLIT_NRMSE
    for c in (0, 31, 32, 39):
        assert nrmse(got[0][:, c], ref[0][:, c]) <= 10 * SPLIT_NRMSE


def test_split_deterministic_and_plan(gpu_context):
    w = W.config(2, spins_stride=200)
    method = BlochHighOrder(w.mask)
    a = split_run(w.obj, w.seq, w.parts, w.excitation, method)
    b = split_run(w.obj, w.seq, w.parts, w.excitation, method)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    params = {"sim_method": method, "precision": "f64", "homs_precision": "split"}
    with homs.prepare_simulation(w.obj, w.seq, sim_params=params, parts=w.parts, excitation=w.excitation) as plan:
        r1 = plan.run()
        r2 = plan.run()
    assert np.array_equal(r1, r2)
    assert np.array_equal(r1[:, :, 0], a[0])


@pytest.mark.parametrize("scenario", ["fixture", "rf", "config1"])
def test_split_fp32_inputs(oracle, gpu_context, scenario):
    # FP32 arrays run on the split path in FP64 and come back as FP32: the
    # signal matches an FP64 computation on the same FP32-rounded inputs to the
    # split bound, and the reference's own FP32 path to its 3e-5 tolerance.
    if scenario == "fixture":
        obj, seq, st = W.high_order_workload(nspins=2000, nsteps=300, ncoils=8)
        parts, exc = [(0, 300)], [False]
    elif scenario == "rf":
        obj, seq, _, _ = W.rf_acquisition_workload(3, 2, 11)
        parts, exc = get_sim_ranges(seq, 4, 5)
        st = None
    else:
        w = W.config(1, spins_stride=41)
        obj, seq, parts, exc, st = w.obj, w.seq, w.parts, w.excitation, None
    method = BlochHighOrder("1111")
    obj32, seq32 = obj.astype(np.float32), seq.astype(np.float32)
    st32 = None if st is None else type(st)(st.xy.astype(np.complex64), st.z.astype(np.float32))
    ref = oracle_run(oracle, obj32.astype(np.float64), seq32.astype(np.float64), parts, exc, method,
                     None if st32 is None else type(st)(st32.xy.astype(np.complex128), st32.z.astype(np.float64)))
    got = homs.run_blocks(obj32, seq32, parts, exc, method, "f32", "split", st32)
    assert got[0].dtype == np.complex64 and got[1].dtype == np.complex64 and got[2].dtype == np.float32
    assert nrmse(got[0], ref[0]) <= SPLIT_NRMSE
    assert nrmse(got[1], ref[1]) <= 1e-6
    assert nrmse(got[2], ref[2]) <= 1e-6
    plain = homs.run_blocks(obj32, seq32, parts, exc, method, "f32", "plain", st32)
    # The plain FP32 kernel accumulates phase in FP32: on the reference's own
    # short fixture it stays within the reference's 3e-5, and over the 10,000
    # samples of a 2D readout it drifts further from the FP64 result than the
    # split path does.
    if scenario == "fixture":
        assert nrmse(got[0], plain[0]) <= 3e-5
    if scenario == "config1":
        assert nrmse(got[0], ref[0]) < nrmse(plain[0], ref[0])


def test_split_fp32_plan_matches_simulate(gpu_context):
    w = W.config(2, spins_stride=400)
    obj32, seq32 = w.obj.astype(np.float32), w.seq.astype(np.float32)
    method = BlochHighOrder(w.mask)
    direct = homs.run_blocks(obj32, seq32, w.parts, w.excitation, method, "f32", "split")
    params = {"sim_method": method, "precision": "f32", "homs_precision": "split"}
    with homs.prepare_simulation(obj32, seq32, sim_params=params, parts=w.parts, excitation=w.excitation) as plan:
        r = plan.run()
    assert r.dtype == np.complex64
    assert np.array_equal(r[:, :, 0], direct[0])


def test_split_phase_range_is_reported(gpu_context):
    # A spin 1 km from the isocentre makes a field term's phase range (largest
    # basis value x largest field integral) exceed 4096 turns in a segment:
    # the split path's fixed-point phase refuses it with HOMS_EUNSUPPORTED.
    obj, seq, st = W.high_order_workload(nspins=33, nsteps=8, ncoils=2)
    obj.x[5] = 1000.0
    with pytest.raises(homs.HomsError) as e:
        homs.run_blocks(obj, seq, [(0, 8)], [False], BlochHighOrder("1111"), "f64", "split", st)
    assert e.value.status == 3
    assert "4096 turns" in str(e.value)
