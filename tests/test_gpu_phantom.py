"""Phantom builders on the GPU against the oracle's restatement of
hophantom_brain / SpinProperty / generate_grid / csm_Birdcage.

The builder rounds every product and sum separately, as the reference does,
so the spin arrays match the oracle bit for bit; the birdcage map goes
through sin/cos/atan2/sqrt and matches to 1e-13."""
import ctypes

import numpy as np
import pytest

import homs
from homs import _lib
from homs.model import BlochHighOrder
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

CLASSES = np.array([23, 46, 70, 93, 116, 139, 162, 185, 209, 232, 255, 0, 0, 3], np.uint8)
FIELDS = ("x", "y", "z", "rho", "T1", "T2", "T2s", "dw")


def _volume(shape, seed, ncoils):
    rng = np.random.default_rng(seed)
    lab = rng.choice(CLASSES, size=shape)
    fm = rng.normal(0, 30, shape)
    csm = (rng.standard_normal(shape + (ncoils,)) + 1j * rng.standard_normal(shape + (ncoils,))) if ncoils else None
    return lab, fm, csm


@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 5, 3), (33, 17, 9), (1, 100, 100), (100, 1, 10), (64, 64, 1)])
@pytest.mark.parametrize("variant", ["fat_unit_1p5T", "fieldmap_csm_7T"])
def test_brain_phantom_matches_oracle(gpu_context, shape, variant):
    fat = variant.startswith("fat")
    fs = "1.5T" if variant.endswith("1p5T") else "7T"
    lab, fm, csm = _volume(shape, sum(shape), 0 if fat else 5)
    res, off = (2e-3, 1.5e-3, 3e-3), (1e-3, -2e-3, 0.5e-3)
    want = orc.brain_phantom_np(lab, res, off, fs, None if fat else fm, csm)
    got = homs.brain_phantom(lab, res, off, fieldstrength=fs, fieldmap=None if fat else fm, csm=csm,
                             context=gpu_context)
    assert len(got) == len(want["x"])
    for k in FIELDS:
        assert np.array_equal(getattr(got, k), want[k]), k
    assert np.array_equal(got.csm, want["csm"])


def test_brain_phantom_device_memory(gpu_context):
    import torch
    lab, fm, csm = _volume((20, 13, 7), 3, 4)
    want = homs.brain_phantom(lab, (2e-3,) * 3, fieldmap=fm, csm=csm, context=gpu_context)
    ns = len(want)
    lab_d = torch.as_tensor(np.asfortranarray(lab).ravel(order="F"), device="cuda:0")
    fm_d = torch.as_tensor(np.asfortranarray(fm).ravel(order="F"), device="cuda:0")
    csm_d = torch.as_tensor(np.asfortranarray(csm).ravel(order="F"), device="cuda:0")
    spec = _lib.BrainSpec()
    spec.nx, spec.ny, spec.nz = lab.shape
    spec.res[:] = [2e-3] * 3
    spec.offcenter[:] = [0.0] * 3
    spec.fieldstrength, spec.ncoils, spec.memory = 0, 4, _lib.HOMS_DEVICE
    spec.labels, spec.fieldmap, spec.csm = lab_d.data_ptr(), fm_d.data_ptr(), csm_d.data_ptr()
    n = ctypes.c_int64()
    lib = _lib.load()
    _lib.check(lib.homs_brain_phantom_count(gpu_context.handle, ctypes.byref(spec), ctypes.byref(n)),
               gpu_context.handle)
    assert n.value == ns
    outs = {k: torch.zeros(ns, dtype=torch.float64, device="cuda:0") for k in FIELDS}
    csm_o = torch.zeros(ns * 4, dtype=torch.complex128, device="cuda:0")
    out = _lib.BrainOut()
    out.nspins, out.memory = ns, _lib.HOMS_DEVICE
    for k, t in outs.items():
        setattr(out, k, t.data_ptr())
    out.csm = csm_o.data_ptr()
    _lib.check(lib.homs_brain_phantom_fill(gpu_context.handle, ctypes.byref(spec), ctypes.byref(out)),
               gpu_context.handle)
    for k in FIELDS:
        assert np.array_equal(outs[k].cpu().numpy(), getattr(want, k)), k
    assert np.array_equal(csm_o.cpu().numpy().reshape(4, ns).T, want.csm)
    out.nspins = ns + 1
    with pytest.raises(homs.HomsError):
        _lib.check(lib.homs_brain_phantom_fill(gpu_context.handle, ctypes.byref(spec), ctypes.byref(out)),
                   gpu_context.handle)


@pytest.mark.parametrize("nx,ny,nc,r", [(64, 64, 8, 1.5), (37, 51, 32, 1.5), (1, 1, 1, 2.0), (100, 80, 12, 1.2)])
def test_birdcage_matches_oracle(gpu_context, nx, ny, nc, r):
    got = homs.csm_birdcage(nx, ny, nc, r, context=gpu_context)
    want = orc.csm_birdcage_np(nx, ny, nc, r)
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))


def test_built_phantom_simulates_like_its_host_copy(oracle, gpu_context):
    # A 2D slice phantom built on the device, with birdcage coils tiled over
    # its single slice, simulated through a resident copy and the oracle.
    from homs import workloads as W
    lab, _, _ = _volume((24, 24, 1), 9, 0)
    coils = homs.csm_birdcage(24, 24, 8, context=gpu_context)[:, :, None, :]
    obj = homs.brain_phantom(lab, (8e-3, 8e-3, 8e-3), csm=coils, context=gpu_context)
    _, seq, _ = W.high_order_workload(nspins=len(obj), nsteps=120, ncoils=8)
    params = {"sim_method": BlochHighOrder("1111"), "precision": "f64", "homs_precision": "plain"}
    state = homs.Mag(np.full(len(obj), 0.3 + 0.4j), obj.rho.copy())
    ref = oracle.simulate_c(obj, seq, [(0, 120)], [False], params["sim_method"].flags, state.xy, state.z)
    got = homs.simulate(obj, seq, sim_params=params, parts=[(0, 120)], excitation=[False], state=state,
                        context=gpu_context)
    assert np.linalg.norm(got[:, :, 0] - ref[0]) <= 1e-12 * np.linalg.norm(ref[0])


@pytest.mark.parametrize("fat", [True, False])
def test_hophantom_brain_from_source_volumes(gpu_context, fat):
    """Source volumes (labels at 0.5 mm, receive and off-resonance maps at
    4 mm) resampled on the host and built on the device, against the oracle
    builder on the same resampled volumes."""
    from homs.phantom import hophantom_brain, resample_b0, resample_csm, resample_labels
    rng = np.random.default_rng(9)
    brain = rng.choice(CLASSES, size=(90, 100, 40))
    b0 = rng.normal(0, 40, (13, 14, 7))
    csm = rng.standard_normal((13, 14, 7, 6)) + 1j * rng.standard_normal((13, 14, 7, 6))
    tres, tmat, loc, off = (2e-3, 2e-3, 2.5e-3), (24, 26, 9), (0.001, -0.002, 0.003), (0.0, 0.0, 1e-3)
    got = hophantom_brain(brain, (0.5e-3,) * 3, tres, tmat, loc, off, b0=None if fat else b0, csm=csm, ncoils=4,
                          context=gpu_context)
    lab = resample_labels(brain, (0.5e-3,) * 3, tres, tmat, loc)
    fm = None if fat else resample_b0(b0, (4e-3,) * 3, tres, tmat, loc)
    cm = resample_csm(csm, (4e-3,) * 3, tres, tmat, loc)[..., :4]
    want = orc.brain_phantom_np(lab, tres, off, "1.5T", fm, cm)
    assert len(got) == len(want["x"]) > 0
    for k in FIELDS:
        assert np.array_equal(getattr(got, k), want[k]), k
    assert np.array_equal(got.csm, want["csm"])
