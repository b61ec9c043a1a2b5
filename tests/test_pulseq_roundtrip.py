"""Randomised round trips through the Pulseq 1.4 reader (CPU, hypothesis): shapes
compressed by the format's rule (derivative, then a value written twice is
followed by the count of further repeats) decode to the original samples, and
random files of trapezoid, arbitrary-gradient and ADC events read back with
the stated units and timing."""
import numpy as np
import pytest

hypothesis = pytest.importorskip("hypothesis")
from hypothesis import given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402

from homs.model import GAMMA  # noqa: E402
from homs.pulseq import decompress_shape, read_seq  # noqa: E402


def _compress(samples):
    """The format's encoding of a shape: run-length over the derivative."""
    d = np.diff(np.concatenate([[0.0], samples]))
    out, i = [], 0
    while i < d.shape[0]:
        j = i
        while j + 1 < d.shape[0] and d[j + 1] == d[i]:
            j += 1
        run = j - i + 1
        if run >= 2:
            out += [d[i], d[i], run - 2]
        else:
            out.append(d[i])
        i = j + 1
    return out


shapes = st.lists(st.tuples(st.integers(-16, 16), st.integers(1, 12)), min_size=1, max_size=12).map(
    lambda runs: np.cumsum(np.concatenate([[v / 8.0] * n for v, n in runs])))


@settings(max_examples=200, deadline=None)
@given(shapes)
def test_shape_compression_round_trip(samples):
    packed = _compress(samples)
    if len(packed) >= samples.shape[0]:
        packed = list(samples)  # a writer stores such shapes uncompressed
    assert np.array_equal(decompress_shape(packed, samples.shape[0]), samples)


@st.composite
def files(draw):
    ntrap = draw(st.integers(1, 4))
    traps = [(i + 1, draw(st.integers(-40, 40)) * 1000, draw(st.integers(0, 30)) * 10, draw(st.integers(1, 80)) * 10,
              draw(st.integers(0, 30)) * 10, draw(st.integers(0, 20)) * 10) for i in range(ntrap)]
    wave = draw(shapes.filter(lambda w: w.shape[0] >= 2))  # an arbitrary gradient has two samples or more
    adcs = [(1, draw(st.integers(1, 64)), draw(st.integers(1, 40)) * 100, draw(st.integers(0, 30)) * 10)]
    blocks = []
    for b in range(draw(st.integers(1, 6))):
        gx = draw(st.integers(0, ntrap + 1))  # id ntrap + 1 is the arbitrary gradient
        gz = draw(st.integers(0, ntrap))
        blocks.append((b + 1, draw(st.integers(100, 300)), 0, gx, 0, gz, draw(st.integers(0, 1)), 0))
    return traps, wave, adcs, blocks


def _write(path, traps, wave, adcs, blocks):
    lines = ["[VERSION]", "major 1", "minor 4", "revision 1", "", "[DEFINITIONS]", "GradientRasterTime 1e-05",
             "BlockDurationRaster 1e-05", "", "[BLOCKS]"]
    lines += [" ".join(str(v) for v in b) for b in blocks]
    lines += ["", "[GRADIENTS]", f"{len(traps) + 1} {GAMMA * 1e-3!r} 1 0 0", "", "[TRAP]"]
    lines += [" ".join(str(v) for v in t) for t in traps]
    lines += ["", "[ADC]"] + [" ".join(str(v) for v in a) + " 0 0" for a in adcs]
    packed = _compress(wave)
    if len(packed) >= wave.shape[0]:
        packed = list(wave)
    lines += ["", "[SHAPES]", "", "shape_id 1", f"num_samples {wave.shape[0]}"] + [repr(float(v)) for v in packed]
    path.write_text("\n".join(lines) + "\n")


@settings(max_examples=60, deadline=None)
@given(files())
def test_random_files_read_back(tmp_path_factory, f):
    traps, wave, adcs, blocks = f
    path = tmp_path_factory.mktemp("seq") / "r.seq"
    _write(path, traps, wave, adcs, blocks)
    seq = read_seq(str(path))
    assert len(seq) == len(blocks)
    tmap = {t[0]: t for t in traps}
    for j, b in enumerate(blocks):
        gx = seq.GR[0, j]
        if b[3] == 0:
            assert not gx.is_on()
        elif b[3] in tmap:
            _, amp, rise, flat, fall, delay = tmap[b[3]]
            assert np.isclose(gx.A, amp / GAMMA, rtol=1e-15, atol=0)
            assert (gx.rise, gx.T, gx.fall, gx.delay) == (rise / 1e6, flat / 1e6, fall / 1e6, delay / 1e6)
        else:
            t, a = gx.knots()
            assert np.allclose(a[1:-1], wave * 1e-3, rtol=1e-15, atol=1e-18)
            assert np.allclose(np.diff(t[1:-1]), 1e-5, rtol=1e-12)
        if b[6]:
            _, num, dwell, delay = adcs[0]
            a = seq.ADC[j]
            assert a.N == num and np.isclose(a.delay, delay / 1e6 + dwell / 2e9, rtol=1e-15)
        events = [g.dur for g in seq.GR[:, j]] + [seq.ADC[j].dur]
        assert np.isclose(seq.DUR[j], max(b[1] * 1e-5, max(events)), rtol=1e-15)
