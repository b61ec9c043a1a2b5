"""The CPU oracle against the reference's known answers, its own NumPy twin,
and the committed golden fixtures (no GPU)."""
import math
import os

import numpy as np
import pytest

from conftest import nrmse
from homs import workloads as W
from homs.model import GAMMA, BlochHighOrder, HO_Phantom

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "oracle_fixtures.npz")


def _run(o, obj, seq, parts, exc, mask, state=None, **kw):
    flags = mask if isinstance(mask, int) else BlochHighOrder(mask).flags
    mxy0 = None if state is None else state.xy
    mz0 = None if state is None else state.z
    return o.simulate_c(obj, seq, parts, exc, flags, mxy0, mz0, **kw)


@pytest.mark.parametrize("ncoils", [1, 3, 32])
@pytest.mark.parametrize("mask", [format(m, "04b") for m in range(16)])
def test_c_oracle_matches_numpy_twin_precession(oracle, mask, ncoils):
    # test/gpu/test_gpu_kernels.jl:16-52 workload, every order mask.
    obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=ncoils)
    flags = BlochHighOrder(mask).flags
    sig_c, xy_c, z_c = oracle.simulate_c(obj, seq, [(0, 32)], [False], flags, st.xy, st.z, nthreads=3)
    sig_n, xy_n, z_n = oracle.simulate_np(obj, seq, [(0, 32)], [False], flags, st.xy, st.z)
    np.testing.assert_allclose(sig_c, sig_n, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(xy_c, xy_n, rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(z_c, z_n, rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("dw_exc", [False, True])
@pytest.mark.parametrize("ncoils", [1, 3, 32])
def test_c_oracle_matches_numpy_twin_excitation(oracle, ncoils, dw_exc):
    # test/gpu/test_gpu_kernels.jl:90-109 workload (RF with ADC on every node).
    obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=ncoils, rf=True)
    flags = BlochHighOrder("1111", dw_exc, True).flags
    sig_c, xy_c, z_c = oracle.simulate_c(obj, seq, [(0, 32)], [True], flags, st.xy, st.z, nthreads=2)
    sig_n, xy_n, z_n = oracle.simulate_np(obj, seq, [(0, 32)], [True], flags, st.xy, st.z)
    np.testing.assert_allclose(sig_c, sig_n, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(xy_c, xy_n, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(z_c, z_n, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("term", range(16))
def test_analytic_phase_per_field_channel(oracle, term):
    # KAT of test/gpu/test_gpu_kernels.jl:54-86: one channel at 2e-5, T1=T2=Inf,
    # dw=0: states = M0 cis(-2 pi gamma b_k(r) 2e-5 t).
    obj, seq, st = W.high_order_workload(nspins=3, nsteps=4, ncoils=3)
    obj.T1[:] = math.inf
    obj.T2[:] = math.inf
    obj.dw[:] = 0
    seq.h[:] = 0
    seq.h[term] = 2e-5
    sig, xy, _ = _run(oracle, obj, seq, [(0, 4)], [False], "1111", st)
    basis = np.stack([oracle.basis_c(x, y, z) for x, y, z in zip(obj.x, obj.y, obj.z)])[:, term]
    phase = -2 * np.pi * GAMMA * basis[:, None] * 2e-5 * seq.t[None, 1:]
    states = st.xy[:, None] * np.exp(1j * phase)
    np.testing.assert_allclose(sig, states.T @ obj.csm, atol=1e-11, rtol=1e-11)
    np.testing.assert_allclose(xy, states[:, -1], atol=1e-11, rtol=1e-11)


def test_ninety_degree_pulse_nominal_only(oracle):
    # KAT of test/unit/test_koma_compatibility.jl:55-69 and :90-97:
    # mask 0000 -> every sample is i*rho^T*csm, final Mxy = i*rho.
    obj = W.compatibility_phantom()
    seq, parts, exc, _ = W.compatibility_sequence()
    sig, xy, _ = _run(oracle, obj, seq, parts, exc, "0000")
    expected = 1j * (obj.rho @ obj.csm)
    assert sig.shape == (5, 2)
    np.testing.assert_allclose(sig, np.repeat(expected[None, :], 5, axis=0), atol=1e-12)
    np.testing.assert_allclose(xy, 1j * obj.rho, atol=1e-12)


def test_zeroth_order_phase_and_rf_ignores_fields(oracle):
    # KAT of test/unit/test_koma_compatibility.jl:118-136: h0 = 20/gamma gives
    # cis(-2 pi 20 t) during readout; a field during RF changes nothing.
    obj = W.compatibility_phantom()
    seq, parts, exc, t_ro = W.compatibility_sequence(h0_readout=20 / GAMMA)
    sig, _, _ = _run(oracle, obj, seq, parts, exc, "1000")
    expected = 1j * (obj.rho @ obj.csm)
    np.testing.assert_allclose(sig, np.exp(-2j * np.pi * 20 * t_ro)[:, None] * expected[None, :], atol=1e-12)
    seq2, parts2, exc2, _ = W.compatibility_sequence(h0_readout=20 / GAMMA, h0_rf=30 / GAMMA)
    sig2, _, _ = _run(oracle, obj, seq2, parts2, exc2, "1000")
    np.testing.assert_allclose(sig2, sig, atol=1e-12)


def test_unit_coil_magnitude_is_total_density(oracle):
    # test/gpu/test_gpu_compatibility.jl:112-114: default coil, pure density ->
    # |signal| = sum(rho) after the 90-degree pulse.
    obj = HO_Phantom(x=[0.0, 0.01, -0.02], rho=[1.0, 0.7, 0.3], T1=[math.inf] * 3, T2=[math.inf] * 3)
    seq, parts, exc, _ = W.compatibility_sequence()
    for term in range(16):
        seq.h[term, 2:] = (term + 1) * 1e-7
    sig, _, _ = _run(oracle, obj, seq, parts, exc, "0000")
    np.testing.assert_allclose(np.abs(sig[:, 0]), obj.rho.sum(), rtol=1e-12)


@pytest.mark.parametrize("block", [1, 2, 32, 128])
def test_block_size_invariance(oracle, block):
    # test/gpu/test_gpu_compatibility.jl:183-187: results do not depend on the
    # block length beyond rounding.
    obj, seq, parts, exc = W.rf_acquisition_workload(3, 2, 11)
    from homs.model import get_sim_ranges
    ref = _run(oracle, obj, seq, parts, exc, "1111")
    p2, e2 = get_sim_ranges(seq, block, max(1, block // 2))
    got = _run(oracle, obj, seq, p2, e2, "1111")
    np.testing.assert_allclose(got[0], ref[0], atol=1e-11, rtol=1e-11)
    np.testing.assert_allclose(got[1], ref[1], atol=1e-11, rtol=1e-11)


def test_reduction_cancellation(oracle):
    # KAT of test/gpu/test_gpu_reduction.jl:55-68.
    states = np.full((4097, 3), 1 - 2j)
    states[1:4096:2] *= -1
    states[-1] = 1e-3 + 2e-3j
    csm = np.full((4097, 3), 0.5 + 0.25j)
    ref = states.T @ csm
    np.testing.assert_allclose(oracle.coil_combine_c(states, csm), ref, atol=1e-14, rtol=0)


def test_golden_fixtures_reproduce(oracle):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    gold = np.load(GOLDEN)
    for name, (obj, seq, parts, exc, mask, st) in mg.cases().items():
        sig, xy, z = _run(oracle, obj, seq, parts, exc, mask, st, nthreads=1)
        np.testing.assert_allclose(sig, gold[f"{name}/sig"], rtol=1e-14, atol=1e-15, err_msg=name)
        np.testing.assert_allclose(xy, gold[f"{name}/xy"], rtol=1e-14, atol=1e-15, err_msg=name)
        np.testing.assert_allclose(z, gold[f"{name}/z"], rtol=1e-14, atol=1e-15, err_msg=name)


def test_thread_count_only_changes_rounding(oracle):
    w = W.config(0, spins_stride=8)
    flags = BlochHighOrder(w.mask).flags
    a = oracle.simulate_c(w.obj, w.seq, w.parts, w.excitation, flags, nthreads=1)
    b = oracle.simulate_c(w.obj, w.seq, w.parts, w.excitation, flags, nthreads=4)
    assert nrmse(b[0], a[0]) < 1e-13
