"""Edge cases: sequences without ADC samples (state-only runs), phantom
volumes without tissue, and the encoding export without ADC times."""
import numpy as np
import pytest

import homs
from conftest import nrmse
from homs import workloads as W
from homs.model import BlochHighOrder, HO_DiscreteSequence, Mag

pytestmark = pytest.mark.gpu


def _no_adc(seq):
    out = HO_DiscreteSequence(seq.t, dt=seq.dt, gx=seq.gx, gy=seq.gy, gz=seq.gz, b1=seq.b1, df=seq.df, psi=seq.psi,
                              adc=np.zeros(seq.nnodes, bool), excitation=seq.excitation, h=seq.h)
    return out


@pytest.mark.parametrize("mode", ["plain", "split"])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_state_only_run_without_adc(oracle, gpu_context, mode, precision):
    obj, seq, st = W.high_order_workload(nspins=700, nsteps=80, ncoils=3)
    seq = _no_adc(seq)
    method = BlochHighOrder("1111")
    ref = oracle.simulate_c(obj, seq, [(0, 80)], [False], method.flags, st.xy, st.z)
    assert ref[0].shape == (0, 3)
    if precision == "f32":
        obj, seq = obj.astype(np.float32), seq.astype(np.float32)
        st = Mag(st.xy.astype(np.complex64), st.z.astype(np.float32))
    params = {"sim_method": method, "precision": precision, "homs_precision": mode, "return_type": "state"}
    got = homs.simulate(obj, seq, sim_params=params, parts=[(0, 80)], excitation=[False], state=st,
                        context=gpu_context)
    tol = 1e-10 if (precision == "f64") else 3e-5
    assert nrmse(got.xy, ref[1]) <= tol and nrmse(got.z, ref[2]) <= tol
    mat = homs.simulate(obj, seq, sim_params=dict(params, return_type="mat"), parts=[(0, 80)], excitation=[False],
                        state=st, context=gpu_context)
    assert mat.shape == (0, 3, 1)


def test_background_only_volume_has_no_spins(gpu_context):
    lab = np.zeros((5, 4, 3), np.uint8)
    lab[1, 1, 1] = 162  # skull: zero density
    obj = homs.brain_phantom(lab, (1e-3,) * 3, context=gpu_context)
    assert len(obj) == 0 and obj.csm.shape == (0, 1)


def test_kspace_without_adc_times(gpu_context):
    w = W.config(0)
    kn, kna, kd, kda = homs.get_kspace(w.seq, adc_times=np.zeros(0), context=gpu_context)
    assert kn.shape == (w.seq.nnodes - 1, 3) and kna.shape == (0, 3) and kda.shape == (0, 16)
