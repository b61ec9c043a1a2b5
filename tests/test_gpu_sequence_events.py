"""Event-level sequences through the engine: the reference's legacy-API and
measured-phase known answers (test/unit/test_koma_compatibility.jl:55-136) run
by ``homs.simulate`` on an ``HO_Sequence``, the generalized encoding export of
an ``HO_Sequence`` (:38-53), and a seeded gradient-echo loop with shaped pulses,
field jumps and measured fields against the FP64 oracle."""
import numpy as np
import pytest

import homs
from conftest import nrmse
from homs import workloads as W
from homs.model import GAMMA, BlochHighOrder, get_sim_ranges
from homs.sequence import ADC, Grad, HO_Sequence, Sequence, discretize, get_adc_sampling_times

pytestmark = pytest.mark.gpu


def test_legacy_simulation_api_and_state_ownership(gpu_context):
    seq = W.compatibility_events()
    hoseq = HO_Sequence(seq)
    obj = W.compatibility_event_phantom()
    density = obj.rho.copy()
    params = {"precision": "f64", "Nthreads": 1, "sim_method": BlochHighOrder("0000"), "return_type": "mat",
              "Nblocks": 1}
    original = dict(params)
    signal = homs.simulate(obj, hoseq, sim_params=params, context=gpu_context)
    expected = 1j * (density @ obj.csm)
    assert signal.shape == (5, 2, 1)
    assert np.allclose(signal[:, :, 0], np.tile(expected, (5, 1)), atol=1e-12, rtol=0)
    assert np.array_equal(obj.rho, density) and params == original
    split = homs.simulate(obj, hoseq, sim_params=dict(params, Nblocks=1000, Nthreads=2), context=gpu_context)
    assert np.allclose(split, signal, atol=1e-12, rtol=0)
    single = homs.simulate(obj, hoseq, sim_params=dict(params, precision="f32"), context=gpu_context)
    assert single.dtype == np.complex64
    assert np.allclose(single, signal, atol=2e-5, rtol=2e-5)
    state = homs.simulate(obj, hoseq, sim_params=dict(params, return_type="state"), context=gpu_context)
    assert isinstance(state, homs.Mag) and state.z is not obj.rho
    assert np.array_equal(obj.rho, density)
    assert np.allclose(state.xy, 1j * density, atol=1e-12, rtol=0)
    raw = homs.simulate(obj, hoseq, sim_params=dict(params, return_type="raw"), context=gpu_context)
    assert sum(p.shape[0] for p in raw.profiles) == 5
    assert all(p.shape[1] == 2 for p in raw.profiles)


@pytest.mark.parametrize("mode,tol", [("plain", 1e-12), ("split", 2e-6)])
def test_measured_zeroth_order_phase(gpu_context, mode, tol):
    seq = W.compatibility_events()
    hoseq = HO_Sequence(seq)
    obj = W.compatibility_event_phantom()
    hoseq.GR_dfc[0, 1] = Grad(20 / GAMMA, 1e-3)
    params = {"precision": "f64", "sim_method": BlochHighOrder("1000"), "return_type": "mat",
              "homs_precision": mode}
    signal = homs.simulate(obj, hoseq, sim_params=params, context=gpu_context)
    expected = 1j * (obj.rho @ obj.csm)
    readout = get_adc_sampling_times(seq) - seq.DUR[0]
    want = np.exp(-2j * np.pi * 20 * readout)[:, None] * expected[None, :]
    assert np.allclose(signal[:, :, 0], want, atol=tol, rtol=0)
    hoseq.GR_dfc[0, 0] = Grad(30 / GAMMA, seq.DUR[0])
    unchanged = homs.simulate(obj, hoseq, sim_params=params, context=gpu_context)
    assert np.allclose(unchanged, signal, atol=tol, rtol=0)


def test_generalized_encoding_output(gpu_context):
    hoseq = HO_Sequence(W.compatibility_events())
    nominal, nominal_adc, measured, measured_adc = homs.get_kspace(hoseq, context=gpu_context)
    assert nominal.shape[1] == 3 and nominal_adc.shape == (5, 3)
    assert measured.shape[1] == 16 and measured_adc.shape == (5, 16)
    assert np.all(nominal_adc == 0) and np.all(measured_adc == 0)


def _gre_case(seed=11, nspins=1500, ncoils=8):
    hoseq = W.gre_events(seed=seed, ntr=3, nadc=48)
    obj, _, _ = W.high_order_workload(nspins=nspins, nsteps=4, ncoils=ncoils)
    return obj, hoseq


@pytest.mark.parametrize("mode,precision,tol", [("plain", "f64", 1e-11), ("split", "f64", 1e-6),
                                                ("plain", "f32", 3e-4), ("split", "f32", 3e-4)])
def test_gre_events_against_the_oracle(oracle, gpu_context, mode, precision, tol):
    obj, hoseq = _gre_case()
    params = {"sim_method": BlochHighOrder("1111"), "precision": precision, "homs_precision": mode, "Δt": 1e-4}
    seqd = discretize(hoseq, sampling_params=params)
    parts, exc = get_sim_ranges(seqd)
    ref, ref_xy, ref_z = oracle.simulate_c(obj, seqd, parts, exc, BlochHighOrder("1111").flags)
    assert ref.shape[0] == 3 * 48
    src = obj if precision == "f64" else obj.astype(np.float32)
    sig = homs.simulate(src, hoseq, sim_params=params, context=gpu_context)
    assert nrmse(sig[:, :, 0], ref) <= tol
    st = homs.simulate(src, hoseq, sim_params=dict(params, return_type="state"), context=gpu_context)
    assert nrmse(st.xy, ref_xy) <= tol and nrmse(st.z, ref_z) <= tol


def test_plan_and_server_take_event_sequences(gpu_context):
    obj, hoseq = _gre_case(seed=12, nspins=900, ncoils=4)
    params = {"sim_method": BlochHighOrder("1111"), "precision": "f64", "homs_precision": "split", "Δt": 2e-4}
    one = homs.simulate(obj, hoseq, sim_params=params, context=gpu_context)
    with homs.prepare_simulation(obj, hoseq, sim_params=params, context=gpu_context) as plan:
        for _ in range(3):
            assert np.array_equal(plan.run(), one)
    with homs.Server(slots=2) as srv:
        ticket = srv.submit(obj, hoseq, sim_params=params)
        assert np.array_equal(srv.result(ticket), one)


def test_adc_phase_compensation_applies_after_the_run(gpu_context):
    obj = W.compatibility_event_phantom()
    base = W.compatibility_events()
    phased = Sequence(base.GR, base.RF, [ADC(0, 0.0), ADC(5, 1e-3, 0.0, 0.0, 0.7)], base.DUR)
    params = {"precision": "f64", "sim_method": BlochHighOrder("0000")}
    a = homs.simulate(obj, HO_Sequence(base), sim_params=params, context=gpu_context)
    b = homs.simulate(obj, HO_Sequence(phased), sim_params=params, context=gpu_context)
    factor = np.complex128(np.complex64(np.exp(-0.7j)))
    assert np.array_equal(b, a * factor)


def test_encoding_export_of_event_sequences(oracle, gpu_context):
    _, hoseq = _gre_case(seed=13)
    seqd, rf_start, rf_sign, adc_times = homs._kspace_inputs(hoseq, 1e-4, None, None, GAMMA)
    assert len(rf_start) == 3 and rf_sign == [0, 0, 0]
    k_ref, kq_ref = oracle.grad2kspace_np(seqd, rf_start, rf_sign, q_times=adc_times)
    kn, kna, km, kma = homs.get_kspace(hoseq, dt=1e-4, context=gpu_context)
    got = np.concatenate([kn, km], axis=1)
    got_q = np.concatenate([kna, kma], axis=1)
    for j in range(19):
        scale = max(np.linalg.norm(k_ref[:, j]), 1e-300)
        assert np.linalg.norm(got[:, j] - k_ref[:, j]) <= 1e-12 * scale
        qs = max(np.linalg.norm(kq_ref[:, j]), 1e-300)
        assert np.linalg.norm(got_q[:, j] - kq_ref[:, j]) <= 1e-12 * qs


def test_callbacks_observe_every_block(gpu_context):
    """test_koma_compatibility.jl:73-81: a callback after every block sees the
    ADC samples done so far, in order, ending at 5; with callbacks the signal
    equals the run without them."""
    hoseq = HO_Sequence(W.compatibility_events())
    obj = W.compatibility_event_phantom()
    params = {"precision": "f64", "Nthreads": 1, "sim_method": BlochHighOrder("0000"), "return_type": "mat",
              "Nblocks": 1}
    signal = homs.simulate(obj, hoseq, sim_params=params, context=gpu_context)
    seen, blocks = [], []

    def callback(progress, info, data, p):
        seen.append(progress.samples - 1)
        blocks.append((progress.block, progress.Nblocks, len(info.parts), data.sig.shape, type(data.Xt).__name__))

    split = homs.simulate(obj, hoseq, sim_params=dict(params, Nblocks=1000, Nthreads=2), context=gpu_context,
                          callbacks=(callback,))
    assert np.allclose(split, signal, atol=1e-12, rtol=0)
    assert seen == sorted(seen) and seen[-1] == 5
    assert [b[0] for b in blocks] == list(range(1, len(blocks) + 1))
    assert all(b[1] == len(blocks) == b[2] and b[3] == (5, 2) and b[4] == "Mag" for b in blocks)
    fields = HO_Sequence(W.compatibility_events())
    fields.GR_dfc[0, 1] = Grad(20 / GAMMA, 1e-3)
    for mode, tol in (("plain", 1e-12), ("split", 2e-6)):
        p = dict(params, sim_method=BlochHighOrder("1111"), homs_precision=mode, Nblocks=3)
        plainrun = homs.simulate(obj, fields, sim_params=p, context=gpu_context)
        withcb = homs.simulate(obj, fields, sim_params=p, context=gpu_context, callbacks=(lambda *a: None,))
        assert np.allclose(withcb, plainrun, atol=tol, rtol=0)
        st = homs.simulate(obj, fields, sim_params=dict(p, return_type="state"), context=gpu_context,
                           callbacks=(lambda *a: None,))
        st0 = homs.simulate(obj, fields, sim_params=dict(p, return_type="state"), context=gpu_context)
        assert np.allclose(st.xy, st0.xy, atol=tol) and np.allclose(st.z, st0.z, atol=tol)
