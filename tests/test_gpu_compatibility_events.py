"""The reference's GPU compatibility tests (test/gpu/test_gpu_compatibility.jl:61-200)
on event-level sequences: the implicit unit receive coil, the high-order
compatibility matrix (precision x orders x coil-combination names) against the
CPU path, and block-length independence with state and raw returns.  The
reference's CPU path is the FP64 oracle on the same discretised sequence."""
import numpy as np
import pytest

import homs
from homs import workloads as W
from homs.model import BlochHighOrder, HO_Phantom, get_sim_ranges
from homs.sequence import Grad, HO_Sequence, discretize

pytestmark = pytest.mark.gpu


def _fields(hoseq):
    for term in range(16):
        hoseq.GR_dfc[term, 1] = Grad((term + 1) * 1e-7, 1e-3)
    return hoseq


def _oracle(oracle, obj, hoseq, orders, params):
    seqd = discretize(hoseq)
    parts, exc = get_sim_ranges(seqd, params.get("max_block_length", np.inf),
                                params.get("max_rf_block_length", np.inf))
    return oracle.simulate_c(obj, seqd, parts, exc, BlochHighOrder(orders).flags)[0]


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("label", ["defaults", "pure density"])
def test_default_receive_coil(oracle, gpu_context, precision, label):
    tol = 3e-5 if precision == "f32" else 1e-11
    inputs = {"x": [0.0, 0.01, -0.02]}
    if label == "pure density":
        inputs.update(rho=[1.0, 0.7, 0.3], T1=[np.inf] * 3, T2=[np.inf] * 3)
    implicit = HO_Phantom(**inputs)
    explicit = HO_Phantom(**inputs, csm=np.ones((3, 1), np.complex128))
    density = implicit.rho.copy()
    hoseq = HO_Sequence(W.compatibility_events())
    if label == "defaults":
        _fields(hoseq)
    params = {"precision": precision, "Nthreads": 1, "sim_method": BlochHighOrder("1111"), "return_type": "mat",
              "max_block_length": 2, "max_rf_block_length": 1}
    reference = _oracle(oracle, explicit, hoseq, "1111", params)
    for combination in homs.HIGH_ORDER_COIL_COMBINATIONS:
        p = dict(params, coil_combination=combination)
        src_i = implicit if precision == "f64" else implicit.astype(np.float32)
        src_e = explicit if precision == "f64" else explicit.astype(np.float32)
        signal = homs.simulate(src_i, hoseq, sim_params=p, context=gpu_context)
        explicit_signal = homs.simulate(src_e, hoseq, sim_params=p, context=gpu_context)
        assert signal.dtype == (np.complex64 if precision == "f32" else np.complex128)
        assert signal.shape == (5, 1, 1) and np.all(np.isfinite(signal))
        assert np.allclose(signal[:, :, 0], reference, atol=tol, rtol=tol)
        assert np.allclose(signal, explicit_signal, atol=tol, rtol=tol)
        if label == "pure density":
            assert np.allclose(np.abs(signal), density.sum(), rtol=tol)
        assert np.array_equal(implicit.rho, density)
        assert np.array_equal(implicit.csm, np.ones((3, 1)))


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("orders", ["0000", "1000", "1111"])
@pytest.mark.parametrize("mode", ["plain", "split"])
def test_high_order_compatibility(oracle, gpu_context, precision, orders, mode):
    hoseq = _fields(HO_Sequence(W.compatibility_events()))
    obj = W.compatibility_event_phantom()
    obj.dw[:] = [5.0, 25.0]
    density = obj.rho.copy()
    params = {"precision": precision, "Nthreads": 1, "sim_method": BlochHighOrder(orders), "return_type": "mat",
              "max_block_length": 2, "max_rf_block_length": 1, "homs_precision": mode}
    reference = _oracle(oracle, obj, hoseq, orders, params)
    tol = 3e-5 if precision == "f32" else (1e-11 if mode == "plain" else 2e-6)
    src = obj if precision == "f64" else obj.astype(np.float32)
    for combination in homs.HIGH_ORDER_COIL_COMBINATIONS:
        signal = homs.simulate(src, hoseq, sim_params=dict(params, coil_combination=combination),
                               context=gpu_context)
        assert np.allclose(signal[:, :, 0], reference, atol=tol, rtol=tol)
        assert np.all(np.isfinite(signal)) and np.array_equal(obj.rho, density)


def test_execution_selection_and_block_lengths(gpu_context):
    obj, hoseq = W.compatibility_event_phantom(), HO_Sequence(W.compatibility_events())
    params = {"precision": "f64", "sim_method": BlochHighOrder("1111"), "return_type": "mat",
              "implementation": "kernel", "max_block_length": 1}
    original = dict(params)
    reference = homs.simulate(obj, hoseq, sim_params=params, context=gpu_context)
    assert params == original
    for block_length in (2, 32, 128):
        signal = homs.simulate(obj, hoseq, sim_params=dict(params, max_block_length=block_length),
                               context=gpu_context)
        assert np.allclose(signal, reference, atol=1e-11, rtol=1e-11)
    for combination in homs.HIGH_ORDER_COIL_COMBINATIONS:
        p = dict(params, coil_combination=combination)
        state = homs.simulate(obj, hoseq, sim_params=dict(p, return_type="state"), context=gpu_context)
        assert np.allclose(state.xy, 1j * obj.rho, atol=1e-11)
        raw = homs.simulate(obj, hoseq, sim_params=dict(p, return_type="raw"), context=gpu_context)
        assert sum(pr.shape[0] for pr in raw.profiles) == 5
        assert all(pr.shape[1] == 2 for pr in raw.profiles)


def test_nominal_bloch_method_agrees_with_the_legacy_path(oracle, gpu_context):
    """test_koma_compatibility.jl:107-115: Bloch() on an HO_Phantom runs the
    nominal gradients only and agrees with the native path; here with
    BlochHighOrder("0000") and with the oracle."""
    hoseq = _fields(HO_Sequence(W.compatibility_events()))
    obj = W.compatibility_event_phantom()
    obj.dw[:] = [5.0, 25.0]
    params = {"precision": "f64", "Nthreads": 1, "return_type": "mat"}
    nominal = homs.simulate(obj, hoseq, sim_params=dict(params, sim_method=homs.Bloch()), context=gpu_context)
    legacy = homs.simulate(obj, hoseq, sim_params=dict(params, sim_method=BlochHighOrder("0000")),
                           context=gpu_context)
    assert np.allclose(nominal, legacy, atol=1e-12, rtol=0)
    seqd = discretize(hoseq)
    parts, exc = get_sim_ranges(seqd)
    ref = oracle.simulate_c(obj, seqd, parts, exc, homs.Bloch().flags)[0]
    assert np.allclose(nominal[:, :, 0], ref, atol=1e-12, rtol=0)


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("rf_limit", [1, np.inf])
@pytest.mark.parametrize("scenario", [(0, 0, 11, True), (3, 2, 11, True), (5, 2, 0, True), (0, 0, 11, False),
                                      (0, 0, 0, True)])
def test_rf_acquisition_through_public_simulate(oracle, gpu_context, precision, rf_limit, scenario):
    """test_gpu_rf_buffers.jl:57-111 on the event-level rf_acquisition_sequence:
    ADC samples during the pulses, every coil-combination name, state and raw."""
    n1, n2, npre, rf_on = scenario
    hoseq = HO_Sequence(W.rf_acquisition_events(n1, n2, npre, rf_on))
    obj = HO_Phantom(x=[-0.01, 0.0, 0.01], y=[0.02, -0.01, 0.0], rho=[1.0, 0.7, 0.2], T1=[0.9, 1.0, 1.1],
                     T2=[0.07, 0.08, 0.09], dw=[-20.0, 5.0, 25.0],
                     csm=np.array([[1, 1j, 0.5], [0.5 - 0.2j, -0.3 + 0.1j, 0.2j], [0.7, 0.2j, 0.4 - 0.3j]]))
    params = {"precision": precision, "implementation": "kernel", "sim_method": BlochHighOrder("1111"),
              "return_type": "mat", "max_block_length": 32, "max_rf_block_length": rf_limit}
    tol = 3e-5 if precision == "f32" else 1e-11
    cpu = _oracle(oracle, obj, hoseq, "1111", params)
    src = obj if precision == "f64" else obj.astype(np.float32)
    reference = homs.simulate(src, hoseq, sim_params=params, context=gpu_context)
    assert reference.shape == (n1 + n2 + npre, 3, 1)
    assert np.allclose(reference[:, :, 0], cpu, atol=tol, rtol=tol)
    ref_state = homs.simulate(src, hoseq, sim_params=dict(params, return_type="state"), context=gpu_context)
    for mode in ("fused_warp", "fused_tiled"):
        p = dict(params, coil_combination=mode)
        owned = dict(p)
        signal = homs.simulate(src, hoseq, sim_params=p, context=gpu_context)
        assert np.allclose(signal, reference, atol=tol, rtol=tol) and np.all(np.isfinite(signal)) and p == owned
        state = homs.simulate(src, hoseq, sim_params=dict(p, return_type="state"), context=gpu_context)
        assert np.array_equal(state.xy, ref_state.xy) and np.array_equal(state.z, ref_state.z)
        if n1 + n2 + npre:
            raw = homs.simulate(src, hoseq, sim_params=dict(p, return_type="raw"), context=gpu_context)
            assert sum(pr.shape[0] for pr in raw.profiles) == n1 + n2 + npre
            assert all(pr.shape[1] == 3 for pr in raw.profiles)
