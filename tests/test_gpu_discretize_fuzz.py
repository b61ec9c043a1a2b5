"""Random event-level sequences (the generators of test_discretize_properties)
simulated by the engine from the HO_Sequence and by the FP64 oracle on the same
discretisation: plain FP64 at 1e-10 and split FP64 at 2e-6 NRMSE."""
import os

import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import HealthCheck, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402

import homs  # noqa: E402
from conftest import nrmse  # noqa: E402
from homs.model import BlochHighOrder, HO_Phantom, get_sim_ranges  # noqa: E402
from homs.sequence import MaxStepSizeRule, discretize, get_adc_sampling_times  # noqa: E402
from test_discretize_properties import sequences  # noqa: E402

pytestmark = pytest.mark.gpu

_RNG = np.random.default_rng(17)
_OBJ = HO_Phantom(x=_RNG.uniform(-0.1, 0.1, 64), y=_RNG.uniform(-0.1, 0.1, 64), z=_RNG.uniform(-0.05, 0.05, 64),
                  rho=_RNG.uniform(0.5, 1.0, 64), T1=_RNG.uniform(0.5, 2.0, 64), T2=_RNG.uniform(0.03, 0.2, 64),
                  dw=_RNG.normal(0, 2 * np.pi * 20, 64),
                  csm=_RNG.standard_normal((64, 2)) + 1j * _RNG.standard_normal((64, 2)))


@settings(max_examples=int(os.environ.get("HOMS_HYPOTHESIS_EXAMPLES", "25")), deadline=None,
          suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large])
@given(sequences(), st.sampled_from(["1111", "0000", "1010"]))
def test_random_event_sequences_match_the_oracle(oracle, gpu_context, hoseq, mask):
    times = get_adc_sampling_times(hoseq.simulation_sequence())
    if times.shape[0] == 0 or np.unique(np.round(times, 13)).shape[0] != times.shape[0]:
        return
    params = {"sim_method": BlochHighOrder(mask), "precision": "f64", "Δt": 1e-4}
    seqd = discretize(hoseq, sampling_rule=MaxStepSizeRule(1e-4, 5e-5))
    parts, exc = get_sim_ranges(seqd)
    ref = oracle.simulate_c(_OBJ, seqd, parts, exc, BlochHighOrder(mask).flags)[0]
    if np.linalg.norm(ref) == 0:
        return
    for mode, tol in (("plain", 1e-10), ("split", 2e-6)):
        got = homs.simulate(_OBJ, hoseq, sim_params=dict(params, homs_precision=mode), context=gpu_context)
        assert nrmse(got[:, :, 0], ref) <= tol, mode
