"""Pulseq 1.4 reading and the reference's demo inputs, on the CPU.

A hand-written file pins the format rules (units, default and shaped timing,
shape compression, signature).  The reference's own demo files, when present
beside this checkout's reference tree, are read and checked against their own
[DEFINITIONS] (total duration, TR, TE, flip angle, ADC size and duration) and
md5 signatures, and the demo loaders (demo3D/1_load_seq.jl,
demo2D/1_load_inputs.jl) are checked for consistent measured fields."""
import hashlib
import math
import os

import numpy as np
import pytest

from homs.model import GAMMA, ArgumentError, BlochHighOrder, count_block_adc, get_sim_ranges
from homs.pulseq import decompress_shape, read_seq, signature_ok
from homs.sequence import HO_Sequence, discretize, get_adc_sampling_times, rf_pulses

# The reference's data files are read only when HOMS_REFERENCE_ROOT names its source tree.
REF = os.environ.get("HOMS_REFERENCE_ROOT", "")
_ref = (lambda *parts: os.path.join(REF, *parts)) if REF else (lambda *parts: "")
N3 = "Spiral_2p0x2p0x2p0_100x100x35_1x4_int1_9p5ms_tr500_te5p0"
SEQ3 = _ref("demo3D", N3 + ".seq")
SEQ2 = _ref("demo2D", "7T_1p0_200_r4.seq")
needs_demo = pytest.mark.skipif(not (os.path.exists(SEQ3) and os.path.exists(SEQ2)),
                                reason="the reference's demo files are not present")


def test_shape_compression():
    samples = np.array([0.0, 1.0, 2.0, 3.0, 4.0, 4.5])
    assert np.array_equal(decompress_shape([0, 1, 1, 2, 0.5], 6), samples)
    assert np.array_equal(decompress_shape(samples, 6), samples)  # listed in full: raw samples
    assert np.array_equal(decompress_shape([0.25, 0.25, 0], 2), [0.25, 0.5])
    with pytest.raises(ArgumentError):
        decompress_shape([0, 1, 1, 5], 5)


_FILE = """# Pulseq sequence file
[VERSION]
major 1
minor 4
revision 1

[DEFINITIONS]
BlockDurationRaster 1e-05
GradientRasterTime 1e-05
RadiofrequencyRasterTime 1e-06
AdcRasterTime 1e-07
FOV 0.2 0.2 0.005
Name unit

# NUM DUR RF  GX  GY  GZ  ADC  EXT
[BLOCKS]
1 120 1 0 0 1 0 0
2 50 0 2 0 0 0 0
3 300 0 3 4 0 1 0

# id amplitude mag_id phase_id time_shape_id delay freq phase
[RF]
1 250 1 2 0 100 12.5 0.5

# id amplitude amp_shape_id time_shape_id delay
[GRADIENTS]
3 1000 3 0 20
4 -2000 4 5 10

# id amplitude rise flat fall delay
[TRAP]
1 4258 100 1000 100 0
2 -8516 50 300 50 0

# id num dwell delay freq phase
[ADC]
1 8 2500 40 0 1.25

[SHAPES]

shape_id 1
num_samples 4
0.5
1
2
3

shape_id 2
num_samples 4
0
0.25
0.5
0.75

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
10
20
"""


def _write(tmp_path, text, sign=True):
    p = tmp_path / "unit.seq"
    body = text.encode()
    if sign:
        body += b"\n[SIGNATURE]\nType md5\nHash " + hashlib.md5(body).hexdigest().encode() + b"\n"
    p.write_bytes(body)
    return str(p)


def test_hand_written_file_events(tmp_path):
    path = _write(tmp_path, _FILE)
    assert signature_ok(path)
    seq = read_seq(path)
    assert len(seq) == 3 and np.allclose(seq.DUR, [1.2e-3, 0.5e-3, 3.0e-3], rtol=1e-15)
    assert seq.DEF["FOV"] == [0.2, 0.2, 0.005] and seq.DEF["Name"] == "unit"
    # trapezoids: Hz/m -> T/m, us -> s
    gz = seq.GR[2, 0]
    assert math.isclose(gz.A, 4258 / GAMMA) and (gz.rise, gz.T, gz.fall) == (1e-4, 1e-3, 1e-4)
    # shaped RF: raw magnitude shape, phase in turns, samples centred in the raster
    rf = seq.RF[0, 0]
    want = 250 / GAMMA * np.array([0.5, 1, 2, 3]) * np.exp(1j * (2 * np.pi * np.array([0, .25, .5, .75]) + 0.5))
    assert np.allclose(rf.A, want, rtol=1e-15) and rf.df == 12.5
    assert math.isclose(rf.delay, 100e-6 + 0.5e-6) and math.isclose(float(np.sum(rf.T)), 3e-6)
    # arbitrary gradient with default timing (compressed shape): samples at (k + 1/2) rasters
    gx = seq.GR[0, 2]
    t, a = gx.knots()
    assert np.allclose(t, 20e-6 + np.array([0, 5, 15, 25, 35, 45, 55, 60]) * 1e-6, rtol=0, atol=1e-18)
    assert np.allclose(a, 1000 / GAMMA * np.array([0, 0, .25, .5, .75, 1, 1.5, 0]), rtol=1e-15)
    # time-shaped gradient: samples at the shape times, first/last from the waveform
    gy = seq.GR[1, 2]
    t, a = gy.knots()
    assert np.allclose(t, 10e-6 + np.array([0, 0, 100, 200, 200]) * 1e-6, rtol=0, atol=1e-18)
    assert np.allclose(a, -2000 / GAMMA * np.array([0, 0, 1, 0, 0]), rtol=1e-15)
    # ADC: samples at delay + (k + 1/2) dwell
    times = get_adc_sampling_times(seq)
    assert np.allclose(times, 1.7e-3 + 40e-6 + (np.arange(8) + 0.5) * 2.5e-6, rtol=0, atol=1e-17)
    assert seq.ADC[2].phi == 1.25
    sd = discretize(HO_Sequence(seq))
    parts, _ = get_sim_ranges(sd)
    assert sum(count_block_adc(sd.adc, parts)) == 8


def test_signature_and_version_checks(tmp_path):
    path = _write(tmp_path, _FILE.replace("Name unit", "Name other"), sign=False)
    assert not signature_ok(path)
    body = _FILE.encode() + b"\n[SIGNATURE]\nType md5\nHash 00000000000000000000000000000000\n"
    p = tmp_path / "bad.seq"
    p.write_bytes(body)
    assert not signature_ok(str(p))
    p2 = tmp_path / "v15.seq"
    p2.write_text(_FILE.replace("minor 4", "minor 5"))
    with pytest.raises(ArgumentError, match="1.4"):
        read_seq(str(p2))
    p3 = tmp_path / "missing.seq"
    p3.write_text(_FILE.replace("3 300 0 3 4 0 1 0", "3 300 0 3 9 0 1 0"))
    with pytest.raises(ArgumentError, match="missing gradient"):
        read_seq(str(p3))


@needs_demo
def test_demo3d_file_matches_its_definitions():
    assert signature_ok(SEQ3)
    seq = read_seq(SEQ3)
    d = seq.DEF
    assert len(seq) == 163
    assert math.isclose(float(np.sum(seq.DUR)), d["TotalDuration"], rel_tol=1e-12)
    nadc = [a.N for a in seq.ADC if a.N]
    assert len(nadc) == d["MatrixSize"][2] and set(nadc) == {int(d["MaxAdcSegmentLength"])}
    a = next(a for a in seq.ADC if a.N)
    dwell = a.T / (a.N - 1)
    assert math.isclose(dwell, d["adcDwell"], rel_tol=1e-12)
    assert math.isclose(a.N * dwell * 1e3, d["adcDuration"], rel_tol=1e-12)
    pulses = rf_pulses(seq)
    assert len(pulses) == 40  # 5 dummy + 35 partitions
    assert all(math.isclose(fa, d["Excit_FlipAngle"], rel_tol=1e-4) for _, fa in pulses)
    assert np.allclose(np.diff([c for c, _ in pulses]), d["TR"], rtol=1e-12)
    first = get_adc_sampling_times(seq)[0] - dwell / 2
    te = [first - c for c, _ in pulses if c < first][-1]
    assert math.isclose(te, d["TE"], rel_tol=1e-9)


@needs_demo
def test_demo2d_file_matches_its_definitions():
    assert signature_ok(SEQ2)
    seq = read_seq(SEQ2)
    d = seq.DEF
    assert sum(a.N for a in seq.ADC) == d["adc_length"]
    a = next(a for a in seq.ADC if a.N)
    assert math.isclose(a.T / (a.N - 1), d["adc_DwellTime"], rel_tol=1e-12)
    pulses = rf_pulses(seq)
    assert len(pulses) == 2 and math.isclose(pulses[1][1], d["flipAngle"], rel_tol=1e-4)
    first = get_adc_sampling_times(seq)[0] - d["adc_DwellTime"] / 2
    assert math.isclose(first - pulses[1][0], d["TE"], rel_tol=1e-9)


@needs_demo
def test_demo_loaders_measured_fields():
    from homs.demo_inputs import demo2d_sequence, demo3d_sequence
    h3 = demo3d_sequence(SEQ3, os.path.join(REF, "demo3D", N3 + ".mat"),
                         os.path.join(REF, "demo3D", N3 + "_skope.mat"))
    sd = discretize(h3)
    parts, _ = get_sim_ranges(sd)
    assert sum(count_block_adc(sd.adc, parts)) == 35 * 3800
    for meas, nom in ((sd.h[1], sd.gx), (sd.h[2], sd.gy)):
        on = nom != 0
        assert np.corrcoef(meas[on], nom[on])[0, 1] > 0.999
    assert all(a.phi == -b.phi for a, b in zip(h3.SEQ.ADC, read_seq(SEQ3).ADC) if a.N)
    h2 = demo2d_sequence(SEQ2, os.path.join(REF, "demo2D", "7T_1p0_200_r4.mat"))
    sd2 = discretize(h2)
    parts, _ = get_sim_ranges(sd2)
    assert len(h2) == 6 and sum(count_block_adc(sd2.adc, parts)) == 29000
    for meas, nom in ((sd2.h[1], sd2.gx), (sd2.h[2], sd2.gy)):
        assert np.corrcoef(meas[sd2.adc], nom[sd2.adc])[0, 1] > 0.999


@needs_demo
def test_demo2d_through_the_oracle(oracle):
    from homs.demo_inputs import demo2d_sequence
    from homs.model import HO_Phantom
    h2 = demo2d_sequence(SEQ2, os.path.join(REF, "demo2D", "7T_1p0_200_r4.mat"))
    sd = discretize(h2)
    parts, exc = get_sim_ranges(sd)
    rng = np.random.default_rng(3)
    n = 16
    obj = HO_Phantom(x=rng.uniform(-0.1, 0.1, n), y=rng.uniform(-0.1, 0.1, n), rho=rng.uniform(0.5, 1, n),
                     T1=np.full(n, 1.0), T2=np.full(n, 0.05), csm=np.ones((n, 1)))
    sig, xy, z = oracle.simulate_c(obj, sd, parts, exc, BlochHighOrder("1111").flags)
    assert sig.shape == (29000, 1) and np.all(np.isfinite(sig))
    assert np.max(np.abs(sig)) <= obj.rho.sum() * (1 + 1e-12)
    nominal, _, _ = oracle.simulate_c(obj, sd, parts, exc, BlochHighOrder("0000").flags)
    # the measured fields follow the nominal gradients: the signals start together and drift apart
    assert abs(sig[0, 0] - nominal[0, 0]) <= 1e-2 * abs(nominal[0, 0])
    assert np.linalg.norm(sig - nominal) > 1e-3 * np.linalg.norm(nominal)


@needs_demo
def test_demo_bench_stage(tmp_path):
    import bench_demo as demo_bench
    phantom_dir = os.path.join(REF, "src", "phantom")
    if not os.path.exists(os.path.join(phantom_dir, "brain3D_0.5_0.5_0.5.mat")):
        pytest.skip("the reference's phantom volumes are not present")
    demo_bench.stage(os.path.join(REF, "demo3D"), phantom_dir, str(tmp_path))
    vol = np.load(tmp_path / "demo3d_phantom_volumes.npz")
    assert vol["labels"].shape == (100, 100, 35) and vol["labels"].dtype == np.uint8
    assert vol["fieldmap"].shape == (100, 100, 35) and np.all(np.isfinite(vol["fieldmap"]))
    assert vol["csm_source"].shape[3] == 32
    assert (vol["labels"] != 0).sum() > 100000
    assert signature_ok(str(tmp_path / (demo_bench.NAME + ".seq")))
    demo_bench.stage(os.path.join(REF, "demo2D"), phantom_dir, str(tmp_path), "demo2d")
    vol2 = np.load(tmp_path / "demo2d_phantom_volumes.npz")
    assert vol2["labels"].shape == (200, 200, 1) and (vol2["labels"] != 0).sum() > 10000
