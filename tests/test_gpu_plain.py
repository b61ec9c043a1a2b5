"""Parity of the plain (FP64/FP32) libhoms kernels with the CPU oracle.

Mirrors the reference's explicit GPU suite (test/gpu/test_gpu_kernels.jl,
test_gpu_reduction.jl, test_gpu_fused_coils.jl, test_gpu_rf_buffers.jl,
test_gpu_compatibility.jl, test_prepared_simulation.jl): kernel vs CPU on
the same fixture, with the reference's tolerances (3e-5 f32, 1e-11 f64) and
the engine's own bar for FP64 (NRMSE <= 1e-12).
"""
import ctypes
import math

import numpy as np
import pytest

import homs
from conftest import nrmse
from homs import _lib
from homs import workloads as W
from homs.model import GAMMA, BlochHighOrder, HO_Phantom, get_sim_ranges

pytestmark = pytest.mark.gpu

TOL = {"f32": 3e-5, "f64": 1e-11}


def oracle_run(o, obj, seq, parts, exc, method, state=None):
    mxy0 = None if state is None else state.xy
    mz0 = None if state is None else state.z
    return o.simulate_c(obj, seq, parts, exc, method.flags, mxy0, mz0)


def gpu_run(obj, seq, parts, exc, method, precision, state=None, mode="plain"):
    return homs.run_blocks(obj, seq, parts, exc, method, precision, mode, state)


def check(got, ref, precision):
    tol = TOL[precision]
    for g, r in zip(got, ref):
        np.testing.assert_allclose(np.asarray(g, np.complex128), r, atol=tol, rtol=tol)
    if precision == "f64":
        assert nrmse(got[0], ref[0]) <= 1e-12
        assert nrmse(got[1], ref[1]) <= 1e-12


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("mask", [format(m, "04b") for m in range(16)])
def test_precession_all_masks(oracle, gpu_context, precision, mask):
    obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=32)
    method = BlochHighOrder(mask, True, True)
    ref = oracle_run(oracle, obj, seq, [(0, 32)], [False], method, st)
    got = gpu_run(obj, seq, [(0, 32)], [False], method, precision, st)
    check(got, ref, precision)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("variant", ["c1", "c3", "no_adc", "no_dw", "c33"])
def test_precession_variants(oracle, gpu_context, precision, variant):
    nc = {"c1": 1, "c3": 3, "c33": 33}.get(variant, 32)
    obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=nc)
    method = BlochHighOrder("1111", True, variant != "no_dw")
    if variant == "no_adc":
        seq.adc[:] = False
    ref = oracle_run(oracle, obj, seq, [(0, 32)], [False], method, st)
    got = gpu_run(obj, seq, [(0, 32)], [False], method, precision, st)
    assert got[0].shape == ref[0].shape
    check(got, ref, precision)


@pytest.mark.parametrize("term", range(16))
def test_analytic_phase_per_field_channel(gpu_context, term):
    # test/gpu/test_gpu_kernels.jl:54-86 on the GPU, f64, closed form at 1e-11.
    obj, seq, st = W.high_order_workload(nspins=3, nsteps=4, ncoils=3)
    obj.T1[:] = math.inf
    obj.T2[:] = math.inf
    obj.dw[:] = 0
    seq.h[:] = 0
    seq.h[term] = 2e-5
    sig, xy, _ = gpu_run(obj, seq, [(0, 4)], [False], BlochHighOrder("1111"), "f64", st)
    x, y, z = obj.x, obj.y, obj.z
    r2 = x ** 2 + y ** 2 + z ** 2
    basis = np.stack([np.ones_like(x), x, y, z, x * y, z * y, 3 * z ** 2 - r2, x * z, x ** 2 - y ** 2,
                      3 * y * x ** 2 - y ** 3, x * z * y, (5 * z ** 2 - r2) * y, 5 * z ** 3 - 3 * z * r2,
                      (5 * z ** 2 - r2) * x, x ** 2 * z - y ** 2 * z, x ** 3 - 3 * x * y ** 2], 1)[:, term]
    states = st.xy[:, None] * np.exp(1j * (-2 * np.pi * GAMMA * basis[:, None] * 2e-5 * seq.t[None, 1:]))
    np.testing.assert_allclose(sig, states.T @ obj.csm, atol=1e-11, rtol=1e-11)
    np.testing.assert_allclose(xy, states[:, -1], atol=1e-11, rtol=1e-11)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("ncoils", [1, 3, 32])
@pytest.mark.parametrize("dw_exc", [False, True])
def test_excitation(oracle, gpu_context, precision, ncoils, dw_exc):
    # test/gpu/test_gpu_kernels.jl:90-109
    obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=ncoils, rf=True)
    method = BlochHighOrder("1111", dw_exc, True)
    ref = oracle_run(oracle, obj, seq, [(0, 32)], [True], method, st)
    got = gpu_run(obj, seq, [(0, 32)], [True], method, precision, st)
    check(got, ref, precision)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_known_answers_through_simulate(gpu_context, precision):
    # test/unit/test_koma_compatibility.jl:55-136 through the public entry point.
    tol = TOL[precision]
    obj = W.compatibility_phantom()
    seq, parts, exc, t_ro = W.compatibility_sequence()
    params = {"sim_method": BlochHighOrder("0000"), "precision": precision, "return_type": "mat"}
    snapshot = dict(params)
    sig = homs.simulate(obj, seq, sim_params=params, parts=parts, excitation=exc)
    assert params == snapshot
    assert sig.shape == (5, 2, 1)
    assert sig.dtype == (np.complex128 if precision == "f64" else np.complex64)
    expected = 1j * (obj.rho @ obj.csm)
    np.testing.assert_allclose(sig[:, :, 0], np.repeat(expected[None], 5, 0), atol=max(tol, 1e-12))
    state = homs.simulate(obj, seq, sim_params={**params, "return_type": "state"}, parts=parts, excitation=exc)
    np.testing.assert_allclose(state.xy, 1j * obj.rho, atol=max(tol, 1e-12))
    seq2, parts2, exc2, t_ro2 = W.compatibility_sequence(h0_readout=20 / GAMMA, h0_rf=30 / GAMMA)
    sig2 = homs.simulate(obj, seq2, sim_params={**params, "sim_method": BlochHighOrder("1000")}, parts=parts2,
                         excitation=exc2)
    np.testing.assert_allclose(sig2[:, :, 0], np.exp(-2j * np.pi * 20 * t_ro2)[:, None] * expected[None],
                               atol=max(tol, 1e-12))
    raw = homs.simulate(obj, seq, sim_params={**params, "return_type": "raw"}, parts=parts, excitation=exc)
    assert sum(p.shape[0] for p in raw.profiles) == 5 and all(p.shape[1] == 2 for p in raw.profiles)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_unit_coil_magnitude(gpu_context, precision):
    # test/gpu/test_gpu_compatibility.jl:61-123 ("pure density")
    obj = HO_Phantom(x=[0.0, 0.01, -0.02], rho=[1.0, 0.7, 0.3], T1=[math.inf] * 3, T2=[math.inf] * 3)
    seq, parts, exc, _ = W.compatibility_sequence()
    sig = homs.simulate(obj, seq, sim_params={"sim_method": BlochHighOrder("1111"), "precision": precision},
                        parts=parts, excitation=exc)
    assert sig.shape == (5, 1, 1)
    np.testing.assert_allclose(np.abs(sig[:, 0, 0]), obj.rho.sum(), rtol=TOL[precision])


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("rf_limit", [1, math.inf])
@pytest.mark.parametrize("scenario", [(0, 0, 11, True), (3, 2, 11, True), (5, 2, 0, True), (0, 0, 11, False),
                                      (0, 0, 0, True)])
def test_rf_acquisition_blocks(oracle, gpu_context, precision, rf_limit, scenario):
    # test/gpu/test_gpu_rf_buffers.jl:195-249: ADC during RF, block limits.
    obj, seq, _, _ = W.rf_acquisition_workload(*scenario)
    parts, exc = get_sim_ranges(seq, 32, rf_limit)
    method = BlochHighOrder("1111")
    ref = oracle_run(oracle, obj, seq, parts, exc, method)
    got = gpu_run(obj, seq, parts, exc, method, precision)
    assert got[0].shape == (scenario[0] + scenario[1] + scenario[2], 3)
    check(got, ref, precision)


@pytest.mark.parametrize("block", [1, 2, 7, 32, 128])
def test_block_length_invariance(gpu_context, block):
    # test/gpu/test_gpu_compatibility.jl:173-187
    obj, seq, st = W.high_order_workload(nspins=300, nsteps=40, ncoils=3)
    method = BlochHighOrder("1111")
    ref = gpu_run(obj, seq, [(0, 40)], [False], method, "f64", st)
    parts, exc = get_sim_ranges(seq, block, block)
    got = gpu_run(obj, seq, parts, exc, method, "f64", st)
    np.testing.assert_allclose(got[0], ref[0], atol=1e-11, rtol=1e-11)
    np.testing.assert_allclose(got[1], ref[1], atol=1e-11, rtol=1e-11)


@pytest.mark.parametrize("nspins", [1, 31, 32, 33, 255, 256, 257, 2051])
def test_spin_tails(oracle, gpu_context, nspins):
    # test/gpu/test_gpu_fused_coils.jl:56-59 tail sizes.
    obj, seq, st = W.high_order_workload(nspins=nspins, nsteps=32, ncoils=3)
    method = BlochHighOrder("1111")
    ref = oracle_run(oracle, obj, seq, [(0, 32)], [False], method, st)
    check(gpu_run(obj, seq, [(0, 32)], [False], method, "f64", st), ref, "f64")


def test_config0_full_fp64(oracle, gpu_context):
    # 4096 spins, 2048 ADC samples, third-order fields: plain FP64 <= 1e-12.
    w = W.config(0)
    method = BlochHighOrder(w.mask)
    ref = oracle_run(oracle, w.obj, w.seq, w.parts, w.excitation, method)
    got = gpu_run(w.obj, w.seq, w.parts, w.excitation, method, "f64")
    assert nrmse(got[0], ref[0]) <= 1e-12
    assert nrmse(got[1], ref[1]) <= 1e-12


@pytest.mark.parametrize("cfg,stride", [(1, 41), (2, 401), (3, 2003)])
def test_config_subsample_fp64(oracle, gpu_context, cfg, stride):
    # Deterministic spin subsamples of the 2D 8-coil, 3D 32-coil and 3D
    # TR-loop workloads (windowed-sinc RF, 35 repetitions): plain FP64 <= 1e-12.
    w = W.config(cfg, spins_stride=stride)
    method = BlochHighOrder(w.mask)
    ref = oracle_run(oracle, w.obj, w.seq, w.parts, w.excitation, method)
    assert np.linalg.norm(ref[0]) > 0
    got = gpu_run(w.obj, w.seq, w.parts, w.excitation, method, "f64")
    assert nrmse(got[0], ref[0]) <= 1e-12
    assert nrmse(got[1], ref[1]) <= 1e-12
    assert nrmse(got[2], ref[2]) <= 1e-12


def _dev(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_block_entry_points_on_device_arrays(oracle, gpu_context, precision):
    # Block-level ABI on caller device memory with a strided signal view and
    # canary rows (test/gpu/test_gpu_kernels.jl:195-218, test_gpu_fused_coils.jl:17-35).
    import torch
    dev = torch.device("cuda:0")
    fdt = torch.float64 if precision == "f64" else torch.float32
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=3)
    lib = _lib.load()
    ctx = gpu_context.handle
    D = lambda a: torch.as_tensor(np.asarray(a), device=dev).to(fdt).contiguous()  # noqa: E731
    px = [D(v) for v in (obj.x, obj.y, obj.z, obj.rho, obj.T1, obj.T2, obj.dw)]
    csm = torch.as_tensor(obj.csm, device=dev).to(cdt).t().contiguous().t()  # column-major
    ph = _lib.Phantom(len(obj), 3, _lib.HOMS_F64 if precision == "f64" else _lib.HOMS_F32, _lib.HOMS_DEVICE,
                      *[t.data_ptr() for t in px], csm.data_ptr())
    nt = len(seq.t)
    sq_arrays = [D(v) for v in (seq.t, seq.dt, seq.gx, seq.gy, seq.gz)]
    b1 = torch.as_tensor(seq.b1, device=dev).to(cdt)
    df, psi = D(seq.df), D(seq.psi)
    adc = torch.as_tensor(seq.adc.astype(np.uint8), device=dev)
    h = D(seq.h)
    hp = (ctypes.c_void_p * 16)(*[h[k].data_ptr() for k in range(16)])
    sq = _lib.Sequence(nt, ph.dtype, _lib.HOMS_DEVICE, *[t.data_ptr() for t in sq_arrays], b1.data_ptr(),
                       df.data_ptr(), psi.data_ptr(), adc.data_ptr(), hp, 0, None, None, None, GAMMA)
    xy = torch.as_tensor(st.xy, device=dev).to(cdt)
    mz = D(st.z)
    state = _lib.State(xy.data_ptr(), mz.data_ptr(), _lib.HOMS_DEVICE)
    parent = torch.full((32 + 4, 3), 7 - 3j, dtype=cdt, device=dev).t().contiguous().t()  # ld = 36
    sig_view = parent[2:34]
    method = BlochHighOrder("1111")
    _lib.check(lib.homs_precession_block(ctx, ctypes.byref(ph), ctypes.byref(sq), 0, 32, method.flags,
                                         ctypes.byref(state), ctypes.c_void_p(sig_view.data_ptr()), 36), ctx)
    torch.cuda.synchronize()
    ref = oracle_run(oracle, obj, seq, [(0, 32)], [False], method, st)
    tol = TOL[precision]
    np.testing.assert_allclose(sig_view.cpu().numpy(), ref[0], atol=tol, rtol=tol)
    np.testing.assert_allclose(xy.cpu().numpy(), ref[1], atol=tol, rtol=tol)
    canary = parent.cpu().numpy()[[0, 1, 34, 35]]
    assert np.all(canary == 7 - 3j)
    # Excitation on the RF fixture, same buffers re-used.
    obj2, seq2, st2 = W.high_order_workload(nspins=259, nsteps=32, ncoils=3, rf=True)
    for t, v in zip(sq_arrays, (seq2.t, seq2.dt, seq2.gx, seq2.gy, seq2.gz)):
        t.copy_(D(v))
    b1.copy_(torch.as_tensor(seq2.b1, device=dev).to(cdt))
    df.copy_(D(seq2.df))
    psi.copy_(D(seq2.psi))
    xy.copy_(torch.as_tensor(st2.xy, device=dev).to(cdt))
    mz.copy_(D(st2.z))
    _lib.check(lib.homs_excitation_block(ctx, ctypes.byref(ph), ctypes.byref(sq), 0, 32, method.flags,
                                         ctypes.byref(state), ctypes.c_void_p(sig_view.data_ptr()), 36), ctx)
    torch.cuda.synchronize()
    ref2 = oracle_run(oracle, obj2, seq2, [(0, 32)], [True], method, st2)
    np.testing.assert_allclose(sig_view.cpu().numpy(), ref2[0], atol=tol, rtol=tol)
    np.testing.assert_allclose(mz.cpu().numpy(), ref2[2], atol=tol, rtol=tol)
    assert np.all(parent.cpu().numpy()[[0, 1, 34, 35]] == 7 - 3j)


def _coil_reduce(ctx, states, csm, precision, ld_pad=4):
    import torch
    dev = torch.device("cuda:0")
    cdt = torch.complex128 if precision == "f64" else torch.complex64
    ns, nadc = states.shape
    nc = csm.shape[1]
    s_t = torch.as_tensor(states, device=dev).to(cdt).t().contiguous().t() if ns and nadc else \
        torch.zeros(1, dtype=cdt, device=dev)
    c_t = torch.as_tensor(csm, device=dev).to(cdt).t().contiguous().t() if ns else torch.zeros(1, dtype=cdt, device=dev)
    parent = torch.full((nc, nadc + ld_pad), 7 - 3j, dtype=cdt, device=dev)  # column-major (nadc+pad) x nc
    sig = parent[:, 2:]
    lib = _lib.load()
    _lib.check(lib.homs_coil_reduce(ctx, _lib.HOMS_F64 if precision == "f64" else _lib.HOMS_F32, ns, nadc, nc,
                                    ctypes.c_void_p(s_t.data_ptr()), max(ns, 1), ctypes.c_void_p(c_t.data_ptr()),
                                    max(ns, 1), ctypes.c_void_p(sig.data_ptr()), nadc + ld_pad), ctx)
    torch.cuda.synchronize()
    full = parent.cpu().numpy()
    return full[:, 2:2 + nadc].T, full


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("nspins", [0, 1, 259, 2049, 32769])
@pytest.mark.parametrize("shape", [(0, 3), (1, 1), (15, 3), (32, 32)])
def test_coil_reduction(gpu_context, precision, nspins, shape):
    # test/gpu/test_gpu_reduction.jl:7-30: normwise error vs FP64 transpose*csm.
    nadc, nc = shape
    rng = np.random.default_rng(42)
    states = rng.standard_normal((nspins, nadc)) + 1j * rng.standard_normal((nspins, nadc))
    csm = rng.standard_normal((nspins, nc)) + 1j * rng.standard_normal((nspins, nc))
    if precision == "f32":
        states = states.astype(np.complex64).astype(np.complex128)
        csm = csm.astype(np.complex64).astype(np.complex128)
    ref = states.T @ csm
    got, full = _coil_reduce(gpu_context.handle, states, csm, precision)
    tol = 5e-6 if precision == "f32" else 5e-13
    scale = max(np.linalg.norm(ref), math.sqrt(nspins * nadc * nc), 1)
    assert np.linalg.norm(got - ref) / scale < tol
    assert np.all(np.isfinite(got))
    assert np.all(full[:, [0, 1, nadc + 2, nadc + 3]] == 7 - 3j)


def test_coil_reduction_many_channels_and_cancellation(gpu_context):
    rng = np.random.default_rng(7)
    states = (rng.standard_normal((1, 257)) + 1j * rng.standard_normal((1, 257))).astype(np.complex64)
    csm = (rng.standard_normal((1, 257)) + 1j * rng.standard_normal((1, 257))).astype(np.complex64)
    got, _ = _coil_reduce(gpu_context.handle, states.astype(np.complex128), csm.astype(np.complex128), "f32")
    ref = states.astype(np.complex128).T @ csm.astype(np.complex128)
    assert np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1) < 5e-6
    # test/gpu/test_gpu_reduction.jl:55-68
    for precision, atol in (("f32", 1e-7), ("f64", 1e-14)):
        st = np.full((4097, 3), 1 - 2j)
        st[1:4096:2] *= -1
        st[-1] = 1e-3 + 2e-3j
        cs = np.full((4097, 3), 0.5 + 0.25j)
        got, _ = _coil_reduce(gpu_context.handle, st, cs, precision)
        np.testing.assert_allclose(got, st.T @ cs, atol=atol, rtol=0)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_prepared_plan_reuse(gpu_context, precision):
    # test/gpu/test_prepared_simulation.jl:5-60: independent runs, snapshots.
    obj, seq, parts, exc = W.rf_acquisition_workload(3, 2, 11)
    params = {"sim_method": BlochHighOrder("1111"), "precision": precision, "max_block_length": 4,
              "max_rf_block_length": 5}
    baseline = homs.simulate(obj, seq, sim_params=params)
    expected_state = homs.simulate(obj, seq, sim_params={**params, "return_type": "state"})
    with homs.prepare_simulation(obj, seq, sim_params=params) as plan:
        first = plan.run()
        assert np.array_equal(first, baseline)
        saved = obj.rho.copy()
        obj.rho *= 2
        assert np.array_equal(plan.run(), baseline)
        obj.rho[:] = saved
        state = plan.run(return_type="state")
        assert np.array_equal(state.xy, expected_state.xy) and np.array_equal(state.z, expected_state.z)
        raw = plan.run(return_type="raw")
        assert sum(p.shape[0] for p in raw.profiles) == 16
        before = first.copy()
        plan.run()
        assert np.array_equal(first, before)
        with pytest.raises(homs.ArgumentError):
            plan.run(return_type="invalid")
        assert plan.device_bytes() > 0
    assert plan.closed
    plan.close()
    with pytest.raises(homs.ArgumentError):
        plan.run()
    # simulate(plan) and the do-block form (PreparedSimulation.jl:181-258)
    got = homs.prepare_simulation(lambda pl: (homs.simulate(pl), homs.simulate(pl, return_type="state"), pl), obj, seq,
                                  sim_params=params)
    assert np.array_equal(got[0], baseline)
    assert np.array_equal(got[1].xy, expected_state.xy) and got[2].closed
    with pytest.raises(homs.ArgumentError):
        homs.simulate(got[2])
    # callbacks on a prepared simulation: after every block, with the same result
    seen = []
    with homs.prepare_simulation(obj, seq, sim_params=params) as plan:
        cb = homs.simulate(plan, callbacks=(lambda pr, info, data, p: seen.append(pr.block),))
        assert np.allclose(cb, baseline, atol=1e-11 if precision == "f64" else 3e-5, rtol=0)
        assert seen == list(range(1, len(plan.parts) + 1))
        st = plan.run(return_type="state", callbacks=(lambda *a: None,))
        assert np.allclose(st.xy, expected_state.xy, atol=1e-11 if precision == "f64" else 3e-5)


def test_prepared_callbacks_failure_edits_and_recursion(gpu_context):
    """test_prepared_simulation.jl:40-61: a failing callback leaves the plan
    and the caller's phantom intact; a callback's state edit reaches the next
    block, as on the one-shot path; recursive use from a callback is refused
    and the plan keeps working."""
    obj, seq, parts, exc = W.rf_acquisition_workload(3, 2, 11)
    density = obj.rho.copy()
    params = {"sim_method": BlochHighOrder("1111"), "precision": "f64", "max_block_length": 4,
              "max_rf_block_length": 5}
    with homs.prepare_simulation(obj, seq, sim_params=params, context=gpu_context) as plan:
        baseline = plan.run()

        def fail(progress, info, data, p):
            data.obj.rho[:] = 0
            data.Xt.xy[:] = 0
            raise RuntimeError("intentional prepared callback failure")

        with pytest.raises(RuntimeError):
            homs.simulate(plan, callbacks=(fail,))
        assert np.array_equal(homs.simulate(plan), baseline) and np.array_equal(obj.rho, density)

        def observe(progress, info, data, p):
            assert np.all(np.isfinite(data.Xt.xy))
            data.Xt.xy *= 1j

        changed = homs.simulate(plan, callbacks=(observe,))
        reference = homs.simulate(obj, seq, sim_params=dict(params, synchronization="block"), callbacks=(observe,),
                                  context=gpu_context)
        assert np.array_equal(changed, reference) and not np.allclose(changed, baseline)
        with pytest.raises(homs.ArgumentError, match="recursively"):
            homs.simulate(plan, callbacks=(lambda *a: homs.simulate(plan),))
        assert np.array_equal(homs.simulate(plan), baseline)
        with pytest.raises(homs.ArgumentError, match="closed from its callback"):
            homs.simulate(plan, callbacks=(lambda *a: plan.close(),))
        assert not plan.closed and np.array_equal(plan.run(), baseline)
    assert plan.closed
