"""A Pulseq file through the engine: the hand-written 1.4 file of the CPU
tests, extended into a small acquisition (shaped excitation, trapezoids,
arbitrary and time-shaped gradients, an ADC window), read, given measured
fields, simulated by the engine and by the FP64 oracle on the same sampled
sequence."""
import numpy as np
import pytest

import homs
from conftest import nrmse
from homs import workloads as W
from homs.model import BlochHighOrder, get_sim_ranges
from homs.pulseq import read_seq
from homs.sequence import Grad, HO_Sequence, discretize

pytestmark = pytest.mark.gpu

_FILE = """[VERSION]
major 1
minor 4
revision 1

[DEFINITIONS]
BlockDurationRaster 1e-05
GradientRasterTime 1e-05
RadiofrequencyRasterTime 1e-06
AdcRasterTime 1e-07

[BLOCKS]
1 120 1 0 0 1 0 0
2 50 0 2 0 0 0 0
3 300 0 3 4 0 1 0
4 80 0 5 0 6 0 0

[RF]
1 30000 1 2 0 100 25 0.3

[GRADIENTS]
3 30000 3 0 20
4 -45000 4 5 10

[TRAP]
1 85000 100 1000 100 0
2 -170000 50 300 50 0
5 200000 100 500 100 0
6 -90000 60 400 60 0

[ADC]
1 200 5000 100 0 0.4

[SHAPES]

shape_id 1
num_samples 9
0.1
0.4
0.8
1
1
0.8
0.4
0.1
0

shape_id 2
num_samples 9
0
0
0
0
0
0
0
0
0

shape_id 3
num_samples 6
0
0.25
0.25
2
0.5

shape_id 4
num_samples 3
0
1
0

shape_id 5
num_samples 3
0
100
200
"""


@pytest.mark.parametrize("mode,tol", [("plain", 1e-11), ("split", 1e-6)])
def test_pulseq_file_through_the_engine(tmp_path, oracle, gpu_context, mode, tol):
    path = tmp_path / "acq.seq"
    path.write_text(_FILE)
    seq = read_seq(str(path))
    hoseq = HO_Sequence(seq)
    rng = np.random.default_rng(21)
    hoseq.GR_dfc[1:4, :] = seq.GR  # measured first order = nominal, plus higher orders below
    for j in range(len(seq)):
        d = float(hoseq.simulation_sequence().DUR[j])
        for i, amp in ((0, 3e-8), (4, 5e-5), (8, 5e-5), (12, 2e-4)):
            hoseq.GR_dfc[i, j] = Grad(amp * rng.standard_normal(7).cumsum(), d)
    obj, _, _ = W.high_order_workload(nspins=800, nsteps=4, ncoils=3)
    params = {"sim_method": BlochHighOrder("1111"), "precision": "f64", "homs_precision": mode, "Δt": 2e-4}
    seqd = discretize(hoseq, sampling_params=params)
    parts, exc = get_sim_ranges(seqd)
    ref, ref_xy, ref_z = oracle.simulate_c(obj, seqd, parts, exc, BlochHighOrder("1111").flags)
    ref = ref * np.complex128(np.complex64(np.exp(-0.4j)))  # the ADC's phase compensation, single-precision factor
    got = homs.simulate(obj, hoseq, sim_params=params, context=gpu_context)
    assert got.shape == (200, 3, 1)
    assert nrmse(got[:, :, 0], ref) <= tol
    st = homs.simulate(obj, hoseq, sim_params=dict(params, return_type="state"), context=gpu_context)
    assert nrmse(st.xy, ref_xy) <= tol and nrmse(st.z, ref_z) <= tol
