"""The comparator that restates the reference's GPU design (materialised states
per block of nodes, cuBLAS coil GEMM; bench.reference_gpu_equivalent) against
the FP64 oracle: on torch's CPU device here, and on the GPU (marked gpu)."""
import pytest

import bench
from conftest import nrmse
from homs import workloads as W
from homs.model import BlochHighOrder


def _cases():
    obj, seq, parts, exc = W.rf_acquisition_workload(3, 2, 11)
    return [("cfg0", W.config(0)), ("rf_acquisition", W.Workload(obj, seq, parts, exc, None, "1111")),
            ("cfg1_sub", W.config(1, spins_stride=200))]


@pytest.mark.parametrize("name,w", _cases(), ids=lambda v: v if isinstance(v, str) else "")
def test_comparator_matches_the_oracle_on_cpu(oracle, name, w):
    ref, _, _ = oracle.simulate_c(w.obj, w.seq, w.parts, w.excitation, BlochHighOrder(w.mask).flags)
    for block in (32, 7):
        got, _ = bench.reference_gpu_equivalent(w, "f64", block, device="cpu", time_it=False)
        assert got.shape == ref.shape and nrmse(got, ref) <= 1e-11
    got32, _ = bench.reference_gpu_equivalent(w, "f32", 32, device="cpu", time_it=False)
    assert nrmse(got32, ref) <= 1e-4


@pytest.mark.gpu
def test_comparator_matches_the_oracle_on_gpu(oracle):
    w = W.config(1, spins_stride=50)
    ref, _, _ = oracle.simulate_c(w.obj, w.seq, w.parts, w.excitation, BlochHighOrder(w.mask).flags)
    got, ms = bench.reference_gpu_equivalent(w, "f64", 32)
    assert ms > 0 and nrmse(got, ref) <= 1e-11
    got32, _ = bench.reference_gpu_equivalent(w, "f32", 32)
    assert nrmse(got32, ref) <= 1e-4
    times = {}
    got_g, ms_g = bench.reference_gpu_equivalent(w, "f64", 32, graph=True, times=times)
    assert ms_g > 0 and times["eager_ms"] > 0 and nrmse(got_g, ref) <= 1e-11
