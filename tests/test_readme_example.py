"""The README's usage example, run as written (test/unit/test_readme_example.jl):
on the GPU through the engine, and on the CPU with ``homs.simulate`` standing
on the FP64 oracle."""
import os
import re

import numpy as np
import pytest

import homs
from conftest import ROOT


def _example() -> str:
    text = open(os.path.join(ROOT, "README.md")).read()
    usage = text.split("## Usage", 1)[1]
    m = re.search(r"```python\n(.*?)\n```", usage, re.S)
    assert m is not None
    return m.group(1)


def _check(signal):
    assert signal.shape == (8, 1, 1) and signal.dtype == np.complex128
    assert np.all(np.isfinite(signal)) and not np.isclose(signal[0, 0, 0], signal[-1, 0, 0])


def test_readme_example_on_the_oracle(oracle, monkeypatch):
    from homs.model import get_sim_ranges
    from homs.sequence import discretize

    def simulate_on_oracle(obj, hoseq, sim_params=None, **kw):
        seqd = discretize(hoseq, sampling_params=sim_params)
        parts, exc = get_sim_ranges(seqd)
        return oracle.simulate_c(obj, seqd, parts, exc, sim_params["sim_method"].flags)[0][:, :, None]

    monkeypatch.setattr(homs, "simulate", simulate_on_oracle)
    scope = {}
    exec(compile(_example(), "README example", "exec"), scope)
    _check(scope["signal"])


@pytest.mark.gpu
def test_readme_example_on_the_gpu():
    scope = {}
    exec(compile(_example(), "README example", "exec"), scope)
    _check(scope["signal"])
