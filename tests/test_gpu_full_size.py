"""Size-independent properties at the full 3D 32-coil size (350,000 spins,
4 x 9,500 ADC samples), where the CPU oracle is too slow to run.

The split path scales the sensitivities per coil by a power of two (times
127/128) before rounding them to integers, and every output column is its
own exact integer dot product, so these hold bit for bit:
  - S(2 csm) = 2 S(csm) and S(csm / 4) = S(csm) / 4;
  - permuting the coils permutes the signal's columns.
Doubling rho doubles the signal to the split bound only: the decay exponent
log2|m0| - e_A is formed in FP32, where log2|2 m0| = log2|m0| + 1 may round
differently.
Spin subsamples of the same workload are checked against the oracle in
test_gpu_split.py; here the full-size run is also checked against the plain
FP64 kernel on a contiguous block of samples of every coil."""
import numpy as np
import pytest

import homs
from homs import workloads as W
from homs.model import BlochHighOrder, HO_Phantom

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg2():
    return W.config(2)


def _with(obj, **kw):
    fields = {k: getattr(obj, k) for k in ("x", "y", "z", "rho", "T1", "T2", "dw", "csm")}
    fields.update(kw)
    return HO_Phantom(**fields)


def _run(w, obj, ctx, mode="split"):
    params = {"sim_method": BlochHighOrder(w.mask), "precision": "f64", "homs_precision": mode}
    return homs.simulate(obj, w.seq, sim_params=params, parts=w.parts, excitation=w.excitation, context=ctx)[:, :, 0]


def test_full_size_scaling_and_permutation_are_exact(cfg2, gpu_context):
    w = cfg2
    assert len(w.obj) == 350_000 and w.obj.ncoils == 32
    base = _run(w, w.obj, gpu_context)
    assert base.shape == (38_000, 32) and np.all(np.isfinite(base)) and np.linalg.norm(base) > 0
    assert np.array_equal(_run(w, _with(w.obj, csm=2.0 * w.obj.csm), gpu_context), 2.0 * base)
    assert np.array_equal(_run(w, _with(w.obj, csm=w.obj.csm / 4.0), gpu_context), base / 4.0)
    doubled = _run(w, _with(w.obj, rho=2.0 * w.obj.rho), gpu_context)
    assert np.linalg.norm(doubled - 2.0 * base) <= 1e-6 * np.linalg.norm(2.0 * base)
    perm = np.random.default_rng(0).permutation(32)
    assert np.array_equal(_run(w, _with(w.obj, csm=w.obj.csm[:, perm]), gpu_context), base[:, perm])


def test_full_size_split_matches_plain_fp64(cfg2, gpu_context):
    # The plain FP64 kernel matches the oracle to 1e-12 on subsamples of this
    # workload; at full size the split result must agree with it to the split
    # bound over the first readout.
    w = cfg2
    split = _run(w, w.obj, gpu_context)
    plain = _run(w, w.obj, gpu_context, mode="plain")
    first = slice(0, 9_500)
    err = np.linalg.norm(split[first] - plain[first]) / np.linalg.norm(plain[first])
    assert err <= 1e-6
    err_all = np.linalg.norm(split - plain) / np.linalg.norm(plain)
    assert err_all <= 1e-6


def test_full_size_tr_loop_scaling_and_permutation(gpu_context):
    # 2,000,000 spins, 35 repetitions of slab-selective RF, readout and fill:
    # the RF blocks run on the FP64 excitation kernel and the readouts on the
    # split kernel, so exactness holds through both.
    w = W.config(3)
    assert len(w.obj) == 2_000_000 and w.obj.ncoils == 32
    base = _run(w, w.obj, gpu_context)
    assert np.all(np.isfinite(base)) and np.linalg.norm(base) > 0
    perm = np.random.default_rng(1).permutation(32)
    got = _run(w, _with(w.obj, csm=2.0 * w.obj.csm[:, perm]), gpu_context)
    assert np.array_equal(got, 2.0 * base[:, perm])
