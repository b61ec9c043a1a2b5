"""Split path beyond one accumulator slot.

The split kernel adds each work item into an int64 accumulator of its tile
and spin-range slot; a slot takes the items whose first 32-spin chunk lies in
one range of 2^18 chunks (8,388,608 spins), and the finalize sums the slots.
8,400,000 spins (262,500 chunks) need two slots.  The CPU oracle is too slow
at this size, so the plain FP64 kernel (itself held to the oracle at 1e-12
by the other tests) is the comparison, at the split path's 1e-6.
"""
import numpy as np
import pytest

import homs
from homs import workloads as W
from homs.model import BlochHighOrder, Mag

from conftest import nrmse

pytestmark = pytest.mark.gpu


def test_split_two_accumulator_slots_match_plain_f64():
    obj, seq, st = W.high_order_workload(nspins=8_400_000, nsteps=8, ncoils=1)
    parts, exc = [(0, 8)], [False]
    m = BlochHighOrder("1111")
    state = Mag(st.xy, st.z)
    plain = homs.run_blocks(obj, seq, parts, exc, m, "f64", "plain", state=state)
    split = homs.run_blocks(obj, seq, parts, exc, m, "f64", "split", state=state)
    assert plain[0].shape == split[0].shape and plain[0].shape[0] == 8
    assert np.abs(plain[0]).max() > 0
    assert nrmse(split[0], plain[0]) <= 1e-6
    # the state update is FP64 in both modes
    assert nrmse(split[1], plain[1]) <= 1e-12
