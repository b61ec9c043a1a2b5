"""Encoding export on the GPU (homs_kspace) against the grad2kspace oracle.

FP64 scan: the GPU sums the trapezoid terms in a different order than the
reference's sequential cumsum, so parity is normwise 1e-12 per column (and
1e-12 of the column's largest value per element)."""
import ctypes

import numpy as np
import pytest

import homs
from homs import _lib
from homs import workloads as W
from homs.model import GAMMA, HO_DiscreteSequence, rf_events
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _check(got, want):
    assert got.shape == want.shape
    for c in range(want.shape[1]):
        w, g = want[:, c], got[:, c]
        scale = float(np.max(np.abs(w))) if w.size else 0.0
        if scale == 0.0:
            assert np.all(g == 0)
            continue
        assert float(np.linalg.norm(g - w)) <= TOL * float(np.linalg.norm(w)) + 1e-300
        assert float(np.max(np.abs(g - w))) <= TOL * scale


def _gpu(seq, starts, signs, q, ctx, precision="f64"):
    kn, kna, kd, kda = homs.get_kspace(seq, rf_start=starts, rf_sign=signs, adc_times=q, context=ctx,
                                       precision=precision)
    return np.hstack([kn, kd]), np.hstack([kna, kda])


@pytest.mark.parametrize("cfg", [0, 1, 3])
def test_kspace_matches_oracle_on_workloads(gpu_context, cfg):
    w = W.config(cfg, spins_stride=10007)
    starts, signs = rf_events(w.seq)
    q = np.asarray(w.seq.t)[np.asarray(w.seq.adc)]
    want_k, want_q = orc.grad2kspace_np(w.seq, starts, signs, GAMMA, q)
    got_k, got_q = _gpu(w.seq, starts, signs, q, gpu_context)
    _check(got_k, want_k)
    _check(got_q, want_q)


def _random_seq(rng, nt, zero_dt=0.05):
    dt = rng.uniform(1e-6, 5e-6, nt - 1)
    dt[rng.random(nt - 1) < zero_dt] = 0.0
    t = np.concatenate([[0.0], np.cumsum(dt)])
    g = rng.standard_normal((3, nt)) * 1e-2
    h = rng.standard_normal((16, nt)) * np.array([1e-6] + [1e-3] * 3 + [5e-3] * 5 + [2e-2] * 7)[:, None]
    return HO_DiscreteSequence(t, dt=dt, gx=g[0], gy=g[1], gz=g[2], h=h)


@pytest.mark.parametrize("nt", [2, 3, 2048, 2049, 2050, 4097, 4098, 20011])
def test_kspace_tails_and_tile_boundaries(gpu_context, nt):
    rng = np.random.default_rng(nt)
    seq = _random_seq(rng, nt)
    m = nt - 1
    cand = sorted({s for s in (1, 2, 2047, 2048, 2049, 4095, 4096, 4097, m - 1) if 1 <= s < m}
                  | set(rng.integers(1, max(m, 2), 5).tolist()) if m > 1 else set())
    cand = [s for s in cand if 1 <= s < m]
    signs = [int(v) for v in rng.integers(-1, 2, len(cand))]
    t = np.asarray(seq.t)
    knots = t[:-1] + np.asarray(seq.dt)
    q = np.concatenate([knots[rng.integers(0, m, 50)], rng.uniform(-1e-5, t[-1] + 1e-5, 50), [knots[0], knots[-1]]])
    want_k, want_q = orc.grad2kspace_np(seq, cand, signs, GAMMA, q)
    got_k, got_q = _gpu(seq, cand, signs, q, gpu_context)
    _check(got_k, want_k)
    _check(got_q, want_q)


def test_kspace_fp32_sequence_arrays(gpu_context):
    # FP32 times accumulated from positive FP32 steps, as a sampled sequence
    # holds them: the knots t[n] + dt[n] are non-decreasing.
    rng = np.random.default_rng(5)
    seq32 = _random_seq(rng, 9000, zero_dt=0.0).astype(np.float32)
    seq32.t = np.concatenate([[np.float32(0)], np.cumsum(seq32.dt, dtype=np.float32)])
    knots = seq32.t[:-1].astype(np.float64) + seq32.dt.astype(np.float64)
    assert np.all(np.diff(knots) >= 0)
    starts, signs = [1000, 5000], [0, -1]
    q = np.asarray(seq32.t, dtype=np.float64)[::7]
    want_k, want_q = orc.grad2kspace_np(seq32.astype(np.float64), starts, signs, GAMMA, q)
    got_k, got_q = _gpu(seq32, starts, signs, q, gpu_context, precision="f32")
    _check(got_k, want_k)
    _check(got_q, want_q)


def test_kspace_linearity_at_full_size(gpu_context):
    # The 3D TR-loop sequence (364,316 nodes, 35 excitations) with the
    # measured first order set to twice the nominal gradients: doubling is
    # exact in floating point, so K_dfc[:, 1:4] == 2 K_nominal bit for bit.
    w = W.config(3, spins_stride=20001)
    seq = w.seq
    seq.h[1:4] = 2 * np.vstack([seq.gx, seq.gy, seq.gz])
    kn, kna, kd, kda = homs.get_kspace(seq, context=gpu_context)
    assert kn.shape == (seq.nnodes - 1, 3) and kd.shape == (seq.nnodes - 1, 16)
    assert np.array_equal(kd[:, 1:4], 2 * kn)
    assert np.array_equal(kda[:, 1:4], 2 * kna)
    ms = ctypes.c_double()
    _lib.check(_lib.load().homs_kspace_timing(gpu_context.handle, ctypes.byref(ms)), gpu_context.handle)
    assert ms.value > 0


def test_kspace_device_memory_matches_host(gpu_context):
    import torch
    rng = np.random.default_rng(11)
    seq = _random_seq(rng, 7000)
    starts = np.array([100, 3000, 6999 - 5], np.int64)
    signs = np.array([0, -1, 1], np.int8)
    q = np.ascontiguousarray(np.asarray(seq.t)[::3])
    host_k, host_q = _gpu(seq, starts.tolist(), signs.tolist(), q, gpu_context)
    dev = {name: torch.as_tensor(np.asarray(getattr(seq, name), np.float64), device="cuda:0")
           for name in ("t", "dt", "gx", "gy", "gz", "df", "psi")}
    h = torch.as_tensor(np.ascontiguousarray(seq.h, np.float64), device="cuda:0")
    b1 = torch.zeros(2 * seq.nnodes, dtype=torch.float64, device="cuda:0")
    adc = torch.zeros(seq.nnodes, dtype=torch.uint8, device="cuda:0")
    hp = (ctypes.c_void_p * 16)(*[h[i].data_ptr() for i in range(16)])
    sq = _lib.Sequence(seq.nnodes, _lib.HOMS_F64, _lib.HOMS_DEVICE, dev["t"].data_ptr(), dev["dt"].data_ptr(),
                       dev["gx"].data_ptr(), dev["gy"].data_ptr(), dev["gz"].data_ptr(), b1.data_ptr(),
                       dev["df"].data_ptr(), dev["psi"].data_ptr(), adc.data_ptr(), hp, 0, None, None, None, GAMMA)
    k = torch.zeros((19, seq.nnodes - 1), dtype=torch.float64, device="cuda:0")  # column-major (m x 19)
    kq = torch.zeros((19, q.shape[0]), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    _lib.check(_lib.load().homs_kspace(gpu_context.handle, ctypes.byref(sq), len(starts), starts.ctypes.data,
                                       signs.ctypes.data, q.shape[0], q.ctypes.data, k.data_ptr(), kq.data_ptr(),
                                       _lib.HOMS_DEVICE), gpu_context.handle)
    assert np.array_equal(k.cpu().numpy().T, host_k)
    assert np.array_equal(kq.cpu().numpy().T, host_q)


def test_kspace_rejects_invalid_breaks(gpu_context):
    seq = _random_seq(np.random.default_rng(2), 100)
    for starts, signs in (([0], [0]), ([99], [0]), ([10, 10], [0, 0]), ([20, 10], [0, 0]), ([10], [2])):
        with pytest.raises(homs.HomsError) as e:
            _gpu(seq, starts, signs, np.zeros(0), gpu_context)
        assert e.value.status == _lib.HOMS_EINVAL
    with pytest.raises(homs.HomsError):
        _gpu(seq, [5], [0], np.array([np.nan]), gpu_context)
