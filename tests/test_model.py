"""Host-side mirror of the reference interface: validation and block planning."""
import numpy as np
import pytest

import homs
from homs import workloads as W
from homs.model import (ArgumentError, BlochHighOrder, DimensionMismatch, HO_Phantom, count_block_adc,
                        get_sim_ranges)


def test_bloch_high_order_mask_rules():
    # src/simulation/BlochHighOrder.jl:21-43
    m = BlochHighOrder("1010")
    assert (m.ho0, m.ho1, m.ho2, m.ho3) == (True, False, True, False)
    assert m.flags == 1 | 4 | 16 | 32
    assert BlochHighOrder("0000", False, True).flags == 32
    for bad in ("111", "11111", "1a11", 1111):
        with pytest.raises(ArgumentError):
            BlochHighOrder(bad)
    with pytest.raises(ArgumentError):
        BlochHighOrder.from_flags(True, True, True, True, name="0111")
    assert BlochHighOrder.from_flags(False, True, True, False).name == "0110"


def test_phantom_defaults_and_validation():
    # src/datatypes/HO_Phantom.jl:47-71, :97-109
    p = HO_Phantom(x=[0.0, 0.01, -0.02])
    assert p.csm.shape == (3, 1) and np.all(p.csm == 1)
    assert np.all(p.rho == 1) and np.all(p.T1 == 1e6)
    p.y = np.zeros(2)
    with pytest.raises(DimensionMismatch):
        p.validate()
    q = HO_Phantom(x=[0.0], csm=np.ones((2, 1)))
    with pytest.raises(DimensionMismatch):
        q.validate()


def test_sim_ranges_share_boundary_nodes_and_own_adc():
    obj, seq, parts, exc = W.rf_acquisition_workload(3, 2, 11)
    p, e = get_sim_ranges(seq)
    assert p == parts and e == exc
    p2, e2 = get_sim_ranges(seq, 1, 1)
    assert all(l - f == 1 for f, l in p2)
    assert sum(count_block_adc(seq.adc, p2)) == sum(count_block_adc(seq.adc, parts)) == 16
    for (f1, l1), (f2, l2) in zip(p2, p2[1:]):
        assert l1 == f2
    with pytest.raises(ArgumentError):
        get_sim_ranges(seq, 0)
    with pytest.raises(ArgumentError):
        get_sim_ranges(seq, 2.5)


def test_setup_validation_matches_reference_errors():
    # src/simulation/Simulate.jl:222-287
    obj = W.compatibility_phantom()
    seq, parts, exc, _ = W.compatibility_sequence()
    setup = homs._setup
    for bad in ({"return_type": "x"}, {"precision": "f16"}, {"synchronization": "x"}, {"implementation": "x"},
                {"coil_combination": "x"}, {"Nthreads": 0}, {"sim_method": "1111"}, {"Nblocks": 0},
                {"max_block_length": 0}, {"implementation": "array"}, {"homs_precision": "bf16"}):
        with pytest.raises(ArgumentError):
            setup(obj, seq, bad)
    with pytest.raises(ArgumentError):
        setup(obj, seq, {1: 2})
    with pytest.raises(ArgumentError):
        setup(obj, seq, [("precision", "f64")])
    params = {"precision": "f64", "Nblocks": 1000}
    snapshot = dict(params)
    p, parts2, exc2 = setup(obj, seq, params)
    assert params == snapshot
    assert all(l - f == 1 for f, l in parts2)
    empty = HO_Phantom(x=np.zeros(0))
    with pytest.raises(ArgumentError):
        setup(empty, seq, {})


def test_config_shapes_and_units():
    w0 = W.config(0)
    assert len(w0.obj) == 4096 and w0.obj.ncoils == 1
    assert sum(count_block_adc(w0.seq.adc, w0.parts)) == 2048
    w1 = W.config(1)
    n1 = sum(count_block_adc(w1.seq.adc, w1.parts))
    assert len(w1.obj) * n1 * w1.obj.ncoils == 40000 * 40000 * 8
    assert w1.mask == "1110"
    # Gradient limit of the spiral readouts.
    g = np.hypot(w1.seq.gx, w1.seq.gy)
    assert g.max() <= 30e-3 * (1 + 1e-9)


def test_config2_size():
    w2 = W.config(2, spins_stride=1000)
    n2 = sum(count_block_adc(w2.seq.adc, w2.parts))
    assert n2 == 4 * 9500 and w2.obj.ncoils == 32
    assert len(W.grid(100, 100, 35, 2e-3, 2e-3, 2e-3)[0]) == 350000


def test_bloch_method_is_accepted_as_nominal_only():
    import homs
    from homs import workloads as W
    from homs.model import Bloch, BlochHighOrder
    seq, parts, exc, _ = W.compatibility_sequence()
    obj = W.compatibility_phantom()
    params, _, _ = homs._setup(obj, seq, {"sim_method": Bloch()})
    assert params["sim_method"] == Bloch() and Bloch().flags == BlochHighOrder("0000").flags
    with pytest.raises(homs.ArgumentError, match="Bloch"):
        homs._setup(obj, seq, {"sim_method": "Bloch"})


def test_basisfunc_spha_terms():
    """basisfunc_spha (basisfunction.jl:24-120): terms 1-16 are the basis the
    simulation uses (the oracle's), and the higher orders are the solid
    harmonics at closed-form points."""
    from homs.sphericalharmonics import basisfunc_spha
    from oracle import oracle as orc
    rng = np.random.default_rng(5)
    x, y, z = rng.uniform(-0.12, 0.12, (3, 50))
    b = basisfunc_spha(x, y, z, list(range(1, 17)))
    assert b.shape == (50, 16)
    assert np.allclose(b, orc.basis_np(x, y, z), rtol=1e-13, atol=1e-18)
    one = np.array([1.0])
    zero = np.array([0.0])
    assert basisfunc_spha(zero, zero, one, 21)[0] == 8.0          # 35 - 30 + 3
    assert basisfunc_spha(one, zero, zero, 36)[0] == 1.0          # x^5
    assert basisfunc_spha(zero, zero, one, 31)[0] == 8.0          # 63 - 70 + 15
    assert basisfunc_spha(one, one, zero, 17)[0] == 0.0           # xy (x^2 - y^2)
    assert basisfunc_spha(x, y, z, [36]).shape == (50, 1)
    from homs.model import ArgumentError
    with pytest.raises(ArgumentError):
        basisfunc_spha(x, y, z, [37])
    assert basisfunc_spha(x.astype(np.float32), y.astype(np.float32), z.astype(np.float32), [2]).dtype == np.float32


def test_phantom_display_defaults_and_container():
    """test_phantom_construction.jl:7-76 and HO_Phantom.jl:74-233: the summary
    string, the ideal default coil and defaults per spin, concatenation and
    density scaling."""
    from homs.model import DimensionMismatch, HO_Phantom
    for dt in (np.float32, np.float64):
        obj = HO_Phantom(x=np.zeros(0, dt), dtype=dt)
        assert repr(obj) == "HO_Phantom[spins | nCoil=1 | nSpin=0 | empty ]" and obj.csm.shape == (0, 1)
        for nc in (0, 2):
            e = HO_Phantom(name="empty", x=np.zeros(0, dt), csm=np.zeros((0, nc)), dtype=dt)
            assert repr(e) == f"HO_Phantom[empty | nCoil={nc} | nSpin=0 | empty ]"
        obj = HO_Phantom(name="display", x=[-0.125, 0.25], y=[0.5, -0.75], z=[-1, 1.5], csm=np.ones((2, 2)),
                         dtype=dt)
        assert repr(obj) == ("HO_Phantom[display | nCoil=2 | nSpin=2 | x=-12.5:25.0 cm | y=-75.0:50.0 cm | "
                             "z=-100.0:150.0 cm ]")
        assert repr(obj[0:0]) == "HO_Phantom[display | nCoil=2 | nSpin=0 | empty ]"
        for n in (0, 1, 3):
            o = HO_Phantom(x=np.zeros(n, dt), dtype=dt)
            assert o.csm.shape == (n, 1) and np.all(o.csm == 1)
            for k in ("y", "z", "dw", "Dlambda1", "Dlambda2", "Dtheta"):
                assert np.array_equal(getattr(o, k), np.zeros(n)) and getattr(o, k).dtype == dt
            assert np.array_equal(o.rho, np.ones(n))
            for k in ("T1", "T2", "T2s"):
                assert np.array_equal(getattr(o, k), np.full(n, 1_000_000.0))
            other = HO_Phantom(x=np.zeros(n, dt), dtype=dt)
            if n:
                o.csm[0, 0] = 0
                assert np.all(other.csm == 1)
    a = HO_Phantom(name="a", x=[0.0, 0.01], rho=[1.0, 0.5], csm=np.ones((2, 3)))
    b = HO_Phantom(name="b", x=[0.02], rho=[0.25], csm=2 * np.ones((1, 3)), Dtheta=[0.3])
    ab = a + b
    assert ab.name == "a+b" and len(ab) == 3 and ab.csm.shape == (3, 3)
    assert np.array_equal(ab.rho, [1.0, 0.5, 0.25]) and np.array_equal(ab.Dtheta, [0, 0, 0.3])
    assert np.array_equal(ab.csm[2], [2, 2, 2])
    with pytest.raises(DimensionMismatch):
        a + HO_Phantom(x=[0.0], csm=np.ones((1, 2)))
    s = 2.0 * a
    assert np.array_equal(s.rho, [2.0, 1.0]) and s.x is a.x and s.allclose(a * 2.0)
    assert not s.allclose(a) and a.allclose(a[0:2])
    assert [len(p) for p in a] == [1, 1]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_phantom_interfaces_and_input_validation(dt):
    """test_phantom_interfaces.jl:7-49: iteration; malformed fields fail with
    DimensionMismatch before any device is touched (simulate and
    prepare_simulation, Bloch() and BlochHighOrder); displacement functions
    follow the concatenation rules and moving phantoms are refused by the
    kernels."""
    import copy as _copy

    import homs
    from homs import workloads as W
    from homs.model import Bloch, BlochHighOrder, DimensionMismatch, HO_Phantom
    from homs.sequence import HO_Sequence
    empty = HO_Phantom(x=np.zeros(0, dt), dtype=dt)
    assert list(empty) == []
    obj = HO_Phantom(x=np.array([0, 0.01, -0.02], dt), dtype=dt)
    assert [s.x[0] for s in obj] == list(obj.x)
    params = {"precision": "f32" if dt == np.float32 else "f64", "Nthreads": 1, "return_type": "mat"}
    hoseq = HO_Sequence(W.compatibility_events())
    for name in ("x", "y", "z", "rho", "T1", "T2", "T2s", "dw", "Dlambda1", "Dlambda2", "Dtheta"):
        bad = _copy.deepcopy(obj)
        setattr(bad, name, np.zeros(2, dt))
        for method in (Bloch(), BlochHighOrder("1111")):
            with pytest.raises(DimensionMismatch):
                homs.simulate(bad, hoseq, sim_params=dict(params, sim_method=method))
        with pytest.raises(DimensionMismatch):
            homs.prepare_simulation(bad, hoseq, sim_params=dict(params, sim_method=BlochHighOrder("1111")))
    for axis in ("ux", "uy", "uz"):
        moving = _copy.deepcopy(obj)

        def displacement(x, y, z, t):
            return t
        setattr(moving, axis, displacement)
        with pytest.raises(homs.ArgumentError):
            obj + moving
        with pytest.raises(homs.ArgumentError):
            moving + obj
        joined = moving + moving
        assert getattr(joined, axis) is displacement and np.array_equal(joined.rho, np.concatenate([moving.rho] * 2))
        assert getattr(empty + moving, axis) is displacement and getattr(moving + empty, axis) is displacement
        with pytest.raises(homs.ArgumentError, match="static"):
            homs.simulate(moving, hoseq, sim_params=dict(params, sim_method=BlochHighOrder("1111")))
