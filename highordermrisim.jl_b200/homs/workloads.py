"""Deterministic workloads: the reference's closed-form fixtures and the
seeded synthetic benchmark configurations.

* ``high_order_workload`` regenerates ``test/support/high_order_workload.jl:4-32``
  (closed-form phantom, sequence and initial state).
* ``compatibility_workload`` / ``rf_acquisition_workload`` give sampled
  versions of ``test/support/compatibility_workload.jl:4-28`` (90-degree hard
  pulse, then a readout; acquisition during RF).  KomaMRI's sampler is not
  vendored, so the node times are chosen here and the known answers are
  computed from them.
* ``config(k)`` builds the seeded synthetic inputs of the five benchmark
  configurations (2D/3D grids, spiral readouts, third-order field waveforms,
  Gaussian receive coils), seeded with PCG64(1000 + k).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

from .model import GAMMA, BlochHighOrder, HO_DiscreteSequence, HO_Phantom, Mag, get_sim_ranges
from .sequence import ADC, RF, Grad, HO_Sequence, Sequence


@dataclass
class Workload:
    obj: HO_Phantom
    seq: HO_DiscreteSequence
    parts: List[Tuple[int, int]]
    excitation: List[bool]
    state: Mag
    mask: str = "1111"
    name: str = ""


def high_order_workload(nspins=32768, nsteps=32, ncoils=32, rf=False):
    """Closed-form fixture of ``test/support/high_order_workload.jl:4-32``.

    Returns (obj, seq, state) for one block of ``nsteps`` intervals with ADC on
    every node but the first.
    """
    u = np.array([0.0]) if nspins == 1 else np.linspace(-1.0, 1.0, nspins)
    coil = np.arange(1, ncoils + 1)[None, :]
    csm = np.exp(1j * (2 * np.pi * coil * u[:, None] / ncoils)) / (1 + coil / ncoils)
    obj = HO_Phantom(x=0.08 * u, y=0.06 * np.sin(3 * u), z=0.04 * np.cos(5 * u), rho=0.8 + 0.2 * np.cos(u),
                     T1=0.9 + 0.1 * np.cos(u), T2=0.07 + 0.01 * np.cos(u), dw=80 * u, csm=csm)
    t = np.linspace(0.0, 2e-4 if rf else 2e-3, nsteps + 1)
    q = np.linspace(0.0, 2 * np.pi, t.shape[0])
    adc = np.ones(t.shape[0], bool)
    adc[0] = False
    h = np.zeros((16, t.shape[0]))
    for term in range(1, 17):
        scale = 1e-7 if term == 1 else 2e-4 if term <= 4 else 1e-3 if term <= 9 else 1e-2
        h[term - 1] = scale * np.sin(q + term / 4)
    seq = HO_DiscreteSequence(
        t, dt=np.diff(t), gx=2e-4 * np.sin(q), gy=2e-4 * np.cos(q), gz=np.full(t.shape[0], 1e-4),
        b1=8e-6 * np.exp(1j * q / 4) if rf else np.zeros(t.shape[0], np.complex128),
        df=100 * np.sin(q) if rf else np.zeros(t.shape[0]),
        psi=0.2 * q if rf else np.zeros(t.shape[0]),
        adc=adc, excitation=np.full(nsteps, rf), h=h)
    state = Mag((0.3 * obj.rho + 1j * 0.6 * obj.rho).astype(np.complex128), 0.5 * obj.rho)
    return obj, seq, state


def compatibility_phantom():
    """Two spins, infinite relaxation, 2-coil CSM (compatibility_workload.jl:17-22)."""
    return HO_Phantom(x=[0.0, 0.01], rho=[1.0, 0.7], T1=[math.inf] * 2, T2=[math.inf] * 2,
                      csm=np.array([[1, 1j], [0.5 - 0.2j, -0.3 + 0.1j]], dtype=np.complex128))


def compatibility_sequence(h0_readout=0.0, h0_rf=0.0, rf_dt=5e-5, readout_dt=2.5e-4, nadc=5):
    """Sampled 90-degree hard pulse (tau = 0.1 ms, B1 = 1/(4 gamma tau)) followed
    by a 2 ms readout block with ``nadc`` samples every ``readout_dt``.

    Returns (seq, parts, excitation, readout_times) where readout_times are
    the ADC times relative to the readout block start.
    """
    tau = 1e-4
    rf_t = np.arange(0.0, tau + 1e-15, rf_dt)
    adc_t = tau + readout_dt * np.arange(1, nadc + 1)
    end = tau + 2e-3
    t = np.concatenate([rf_t, adc_t, [end]])
    nt = t.shape[0]
    nrf = rf_t.shape[0]
    b1 = np.zeros(nt, np.complex128)
    b1[:nrf - 1] = 1.0 / (4 * GAMMA * tau)
    adc = np.zeros(nt, bool)
    adc[nrf:nrf + nadc] = True
    exc = np.zeros(nt - 1, bool)
    exc[:nrf - 1] = True
    h = np.zeros((16, nt))
    h[0, :nrf] = h0_rf
    h[0, nrf - 1:] = h0_readout
    seq = HO_DiscreteSequence(t, dt=np.diff(t), b1=b1, adc=adc, excitation=exc, h=h)
    parts = [(0, nrf - 1), (nrf - 1, nt - 1)]
    return seq, parts, [True, False], adc_t - tau


def rf_acquisition_workload(nrf_first=3, nrf_last=2, npre=11, rf_on=True):
    """Sampled restatement of ``rf_acquisition_sequence`` (compatibility_workload.jl:30-39):
    RF (tau = 120 us) with acquisition, a 2 ms readout block, and a second RF
    with acquisition.  Returns (obj, seq, parts, excitation)."""
    tau = 120e-6
    a1 = 1 / (4 * GAMMA * tau) if rf_on else 0.0
    a2 = 1 / (8 * GAMMA * tau) if rf_on else 0.0

    def rf_block(t0, n, amp):
        base = np.linspace(0.0, tau, 5)
        adc_t = tau / 4 + (tau / 2) * (np.arange(n) / max(n - 1, 1)) if n > 1 else (
            np.array([tau / 2]) if n == 1 else np.zeros(0))
        tt = np.unique(np.concatenate([base, adc_t]))
        adc = np.isin(tt, adc_t)
        return t0 + tt, adc, np.full(tt.shape[0], amp, np.complex128)

    t1, adc1, b11 = rf_block(0.0, nrf_first, a1)
    pre_t = tau + (1e-3 + 1e-4 * np.arange(npre)) if npre else np.zeros(0)
    t2 = np.concatenate([[tau], pre_t, [tau + 2e-3]])
    adc2 = np.concatenate([[False], np.ones(npre, bool), [False]])
    t3, adc3, b13 = rf_block(tau + 2e-3, nrf_last, a2)
    t = np.concatenate([t1, t2[1:], t3[1:]])
    adc = np.concatenate([adc1, adc2[1:], adc3[1:]])
    b1 = np.concatenate([b11, np.zeros(t2.shape[0] - 1, np.complex128), b13[1:]])
    n1 = t1.shape[0]
    n2 = n1 + t2.shape[0] - 1
    exc = np.zeros(t.shape[0] - 1, bool)
    exc[:n1 - 1] = True
    exc[n2 - 1:] = True
    b1[n1 - 1] = 0.0
    b1[-1] = 0.0
    seq = HO_DiscreteSequence(t, dt=np.diff(t), b1=b1, adc=adc, excitation=exc)
    obj = HO_Phantom(x=[-0.01, 0.0, 0.01], y=[0.02, -0.01, 0.0], rho=[1.0, 0.7, 0.2], T1=[0.9, 1.0, 1.1],
                     T2=[0.07, 0.08, 0.09], dw=[-20.0, 5.0, 25.0],
                     csm=np.array([[1, 1j, 0.5], [0.5 - 0.2j, -0.3 + 0.1j, 0.2j], [0.7, 0.2j, 0.4 - 0.3j]]))
    parts = [(0, n1 - 1), (n1 - 1, n2 - 1), (n2 - 1, t.shape[0] - 1)]
    return obj, seq, parts, [True, False, True]


# ---------------------------------------------------------------------------
# Event-level sequences (HO_Sequence built from Grad / RF / ADC events)
# ---------------------------------------------------------------------------

def compatibility_events():
    """Event-level ``compatibility_sequence`` (test/support/compatibility_workload.jl:4-10):
    a 90-degree hard pulse of 0.1 ms, then a 2 ms block with 5 ADC samples over 1 ms."""
    rf_duration = 1e-4
    gradients = [[Grad(0.0, 0.0), Grad(0.0, 0.0)] for _ in range(3)]
    pulses = [RF(1 / (4 * GAMMA * rf_duration), rf_duration), RF(0.0, 0.0)]
    adc = [ADC(0, 0.0), ADC(5, 1e-3)]
    return Sequence(gradients, pulses, adc, [rf_duration, 2e-3])


def compatibility_event_phantom():
    """``compatibility_phantom`` (compatibility_workload.jl:12-18)."""
    return HO_Phantom(x=[0.0, 0.01], rho=[1.0, 0.7], T1=[math.inf] * 2, T2=[math.inf] * 2,
                      csm=np.array([[1, 1j], [0.5 - 0.2j, -0.3 + 0.1j]]))


def rf_acquisition_events(nrf_first, nrf_last, npre, rf_on=True):
    """Event-level ``rf_acquisition_sequence`` (compatibility_workload.jl:20-28): RF
    pulses of 120 us that acquire during the pulse, around a 2 ms block."""
    tau = 120e-6
    gradients = [[Grad(0.0, 0.0)] * 3 for _ in range(3)]
    a1 = 1 / (4 * GAMMA * tau) if rf_on else 0.0
    a2 = 1 / (8 * GAMMA * tau) if rf_on else 0.0
    pulses = [RF(a1, tau), RF(0.0, 0.0), RF(a2, tau)]

    def rf_adc(n):
        return ADC(0, 0.0) if n == 0 else ADC(n, tau / 2, tau / 4)

    adcs = [rf_adc(nrf_first), ADC(0, 0.0) if npre == 0 else ADC(npre, 1e-3, 1e-4), rf_adc(nrf_last)]
    return Sequence(gradients, pulses, adcs, [tau, 2e-3, tau])


def gre_events(seed=7, ntr=3, nadc=64, dwell=4e-6, flip_deg=30.0, tr=12e-3, field_scale=1.0):
    """Seeded gradient-echo TR loop as events: a windowed-sinc slab pulse on a
    slice-select trapezoid (zero-rise edges included, so field jumps occur),
    phase/readout prewinders, a readout trapezoid with its ADC, spoilers, and
    measured high-order fields as sampled ``Grad`` waveforms (h0, the first
    order rows, and a few second and third order rows) over every block.
    Returns an ``HO_Sequence``."""
    rng = np.random.default_rng(seed)
    seq = None
    gr_cols = []
    for r in range(ntr):
        # excitation: 1.6 ms sinc (time-bandwidth 4) on a flat slice gradient with
        # a zero-rise start and a 0.2 ms ramp down
        n = 33
        x = np.linspace(-2, 2, n)
        shape = np.sinc(x) * (0.54 + 0.46 * np.cos(np.pi * x / 2))
        dur = 1.6e-3
        area = np.sum((shape[1:] + shape[:-1]) / 2) * dur / (n - 1)
        amp = np.deg2rad(flip_deg) / (2 * np.pi * GAMMA * area)
        phase = np.exp(1j * np.pi * r * (r + 1) / 2 * 117 / 180)  # RF spoiling
        rf = RF(amp * shape * phase, dur, df=float(rng.uniform(-50, 50)), delay=0.1e-3)
        ss = Grad(8e-3, 1.8e-3, 0.0, 2e-4)
        b_exc = Sequence([[Grad(0.0, 0.0)], [Grad(0.0, 0.0)], [ss]], [rf], [ADC(0, 0.0)])
        # prewinders: readout, phase encoding, slice refocusing
        ky = (r - ntr / 2) / max(ntr, 1)
        pre = Sequence([[Grad(-6e-3, 0.4e-3, 1e-4)], [Grad(10e-3 * ky, 0.4e-3, 1e-4)], [Grad(-9e-3, 0.3e-3, 1e-4)]])
        # readout with its ADC centred on the flat top
        ro_T = nadc * dwell
        ro = Sequence([[Grad(6e-3, ro_T, 1e-4)], [Grad(0.0, 0.0)], [Grad(0.0, 0.0)]], None,
                      [ADC(nadc, ro_T - dwell, 1e-4 + dwell / 2)])
        spoil = Sequence([[Grad(12e-3, 1e-3, 2e-4)], [Grad(-10e-3 * ky, 0.4e-3, 1e-4)], [Grad(15e-3, 1e-3, 2e-4)]])
        block = b_exc + pre + ro + spoil
        fill = tr - float(np.sum(block.DUR))
        block = block + Sequence([[Grad(0.0, 0.0)]] * 3, None, None, [max(fill, 0.0)])
        seq = block if seq is None else seq + block
    # measured fields: a smooth random waveform per (channel, block), nominal-like in rows 1-3
    rows = [0, 1, 2, 3, 4, 6, 8, 9, 12]
    amps = {0: 2e-7, 1: 4e-5, 2: 4e-5, 3: 4e-5, 4: 2e-4, 6: 2e-4, 8: 2e-4, 9: 1e-3, 12: 1e-3}
    nominal = {1: 0, 2: 1, 3: 2}
    gr = np.empty((16, len(seq)), dtype=object)
    for j in range(len(seq)):
        D = float(seq.DUR[j])
        for i in range(16):
            if i in rows and D > 0:
                ns = 9
                a = field_scale * amps[i] * rng.standard_normal(ns).cumsum() / 3
                if i in nominal:  # measured first order: the nominal waveform's area plus a perturbation
                    g = seq.GR[nominal[i], j]
                    a = a + (g.area() / D if D > 0 else 0.0)
                gr[i, j] = Grad(a, D)
            else:
                gr[i, j] = Grad(0.0, 0.0)
    return HO_Sequence(seq, gr)


# ---------------------------------------------------------------------------
# Seeded synthetic benchmark configurations
# ---------------------------------------------------------------------------

def grid(nx, ny, nz, dx, dy, dz):
    """Centred grid with x fastest (``src/grid/Grid.jl:36-39``)."""
    i = np.arange(1, nx + 1) - (nx + 1) / 2
    j = np.arange(1, ny + 1) - (ny + 1) / 2
    k = np.arange(1, nz + 1) - (nz + 1) / 2
    zz, yy, xx = np.meshgrid(k, j, i, indexing="ij")
    return xx.ravel() * dx, yy.ravel() * dy, zz.ravel() * dz


def tissue(rng, n, sigma_hz):
    rho = rng.uniform(0.5, 1.0, n)
    T1 = rng.uniform(0.5, 2.0, n)
    T2 = rng.uniform(0.03, 0.2, n)
    dw = 2 * np.pi * rng.normal(0.0, sigma_hz, n)
    return rho, T1, T2, dw


def gaussian_coils(rng, x, y, z, centres, sigma):
    phase = rng.uniform(0, 2 * np.pi, centres.shape[0])
    d2 = ((x[:, None] - centres[None, :, 0]) ** 2 + (y[:, None] - centres[None, :, 1]) ** 2 +
          (z[:, None] - centres[None, :, 2]) ** 2)
    return np.exp(-d2 / (2 * sigma ** 2)) * np.exp(1j * phase)[None, :]


def fibonacci_hemisphere(n, radius):
    k = np.arange(n) + 0.5
    zc = k / n
    r = np.sqrt(1 - zc ** 2)
    phi = np.pi * (1 + 5 ** 0.5) * k
    return np.stack([radius * r * np.cos(phi), radius * r * np.sin(phi), radius * zc], axis=1)


def spiral_gradients(nsamples, dwell, kmax, gmax, rotation=0.0):
    """Archimedean spiral k(t) = kmax (t/T) exp(i(2 pi n t/T + rot)); the number
    of turns is chosen so that max |G| equals gmax.  Returns (gx, gy) in T/m
    at the sample times t = dwell, 2 dwell, ..."""
    T = nsamples * dwell
    t = dwell * np.arange(1, nsamples + 1)
    turns = 1.0
    for _ in range(60):  # fixed-point solve for the turn count that meets gmax
        w = 2 * np.pi * turns / T
        kr = kmax * t / T
        dk = kmax / T * np.exp(1j * (w * t + rotation)) + 1j * w * kr * np.exp(1j * (w * t + rotation))
        g = np.max(np.abs(dk)) / GAMMA
        turns *= gmax / g
    w = 2 * np.pi * turns / T
    kr = kmax * t / T
    dk = kmax / T * np.exp(1j * (w * t + rotation)) + 1j * w * kr * np.exp(1j * (w * t + rotation))
    g = dk / GAMMA
    return g.real, g.imag


def field_waveforms(rng, t, amplitudes):
    """16 x Nt coefficients: each term a sum of 3 seeded sinusoids (50-500 Hz);
    ``amplitudes`` gives the per-order bound (T, T/m, T/m^2, T/m^3)."""
    h = np.zeros((16, t.shape[0]))
    order = [0] + [1] * 3 + [2] * 5 + [3] * 7
    for k in range(16):
        a = amplitudes[order[k]] / 3
        for _ in range(3):
            f = rng.uniform(50, 500)
            ph = rng.uniform(0, 2 * np.pi)
            h[k] += a * rng.uniform(0.5, 1.0) * np.sin(2 * np.pi * f * t + ph)
    return h


class _SeqBuilder:
    """Appends sampled sections; adjacent sections share their boundary node."""

    def __init__(self):
        self.t = [0.0]
        self.gx, self.gy, self.gz = [0.0], [0.0], [0.0]
        self.b1 = [0j]
        self.adc = [False]
        self.exc: List[bool] = []

    def add(self, dts, gx=None, gy=None, gz=None, b1=None, adc=None, excitation=False):
        n = len(dts)
        gx = np.zeros(n) if gx is None else gx
        gy = np.zeros(n) if gy is None else gy
        gz = np.zeros(n) if gz is None else gz
        b1 = np.zeros(n, np.complex128) if b1 is None else b1
        adc = np.zeros(n, bool) if adc is None else adc
        t = self.t[-1]
        for i in range(n):
            t = t + dts[i]
            self.t.append(t)
        self.gx.extend(gx)
        self.gy.extend(gy)
        self.gz.extend(gz)
        self.b1.extend(b1)
        self.adc.extend(adc)
        self.exc.extend([excitation] * n)

    def hard_rf(self, flip_deg, tau=1e-4, dt=5e-5):
        """Hard pulse: B1 constant on the interval start nodes of the pulse."""
        n = int(round(tau / dt))
        amp = (flip_deg / 360.0) / (GAMMA * tau)
        self.b1[-1] = amp
        b1 = np.full(n, amp, np.complex128)
        b1[-1] = 0.0
        self.add(np.full(n, dt), b1=b1, excitation=True)

    def build(self, h_fn):
        t = np.asarray(self.t)
        h = h_fn(t)
        seq = HO_DiscreteSequence(t, dt=np.diff(t), gx=np.asarray(self.gx), gy=np.asarray(self.gy),
                                  gz=np.asarray(self.gz), b1=np.asarray(self.b1), adc=np.asarray(self.adc),
                                  excitation=np.asarray(self.exc), h=h)
        return seq


CONFIG_NAMES = {
    0: "2d_spiral_64x64_4096spins_1coil_f64",
    1: "2d_spiral_200x200_40000spins_8coils_4x10000adc",
    2: "3d_stack_of_spirals_100x100x35_350000spins_32coils_4x9500adc",
    3: "3d_tr_loop_200x200x50_2000000spins_32coils_35tr_9500adc",
}


def config(k: int, max_block_length=math.inf, spins_stride: int = 1) -> Workload:
    """Seeded synthetic inputs of benchmark configuration ``k`` (0-3).

    ``spins_stride`` keeps every n-th spin (a deterministic subsample used for
    bounded CPU-oracle runs)."""
    rng = np.random.Generator(np.random.PCG64(1000 + k))
    amps = (1e-6, 1e-3, 5e-3, 20e-3)
    if k == 0:
        x, y, z = grid(64, 64, 1, 0.2 / 64, 0.2 / 64, 1.0)
        z = np.zeros_like(x)
        rho, T1, T2, dw = tissue(rng, x.shape[0], 20.0)
        rho = rho * ((x ** 2 + y ** 2) <= 0.09 ** 2)
        csm = np.ones((x.shape[0], 1), np.complex128)
        b = _SeqBuilder()
        b.hard_rf(90.0)
        gx, gy = spiral_gradients(2048, 5e-6, 64 / (2 * 0.2), 30e-3)
        b.add(np.full(2048, 5e-6), gx=gx, gy=gy, adc=np.ones(2048, bool))
        mask = "1111"
    elif k == 1:
        x, y, z = grid(200, 200, 1, 1e-3, 1e-3, 1.0)
        z = np.zeros_like(x)
        rho, T1, T2, dw = tissue(rng, x.shape[0], 50.0)
        rho = rho * ((x ** 2 + y ** 2) <= 0.09 ** 2)
        ang = 2 * np.pi * np.arange(8) / 8
        centres = np.stack([0.15 * np.cos(ang), 0.15 * np.sin(ang), np.zeros(8)], axis=1)
        csm = gaussian_coils(rng, x, y, z, centres, 0.08)
        b = _SeqBuilder()
        for il in range(4):
            b.hard_rf(90.0)
            gx, gy = spiral_gradients(10000, 1e-6, 200 / (2 * 0.2), 30e-3, rotation=il * np.pi / 2)
            b.add(np.full(10000, 1e-6), gx=gx, gy=gy, adc=np.ones(10000, bool))
        mask = "1110"
    elif k in (2, 3):
        if k == 2:
            nx, ny, nz, d, sig_hz, nil, nro = 100, 100, 35, 2e-3, 80.0, 4, 9500
        else:
            nx, ny, nz, d, sig_hz, nil, nro = 200, 200, 50, 1e-3, 80.0, 35, 9500
        x, y, z = grid(nx, ny, nz, d, d, d)
        rho, T1, T2, dw = tissue(rng, x.shape[0], sig_hz)
        ax, ay, az = 0.45 * nx * d, 0.45 * ny * d, 0.45 * nz * d
        rho = rho * (((x / ax) ** 2 + (y / ay) ** 2 + (z / az) ** 2) <= 1.0)
        centres = fibonacci_hemisphere(32, 0.14)
        csm = gaussian_coils(rng, x, y, z, centres, 0.08)
        b = _SeqBuilder()
        fovz = nz * d
        for il in range(nil):
            if k == 2:
                b.hard_rf(90.0)
            else:
                _windowed_sinc_rf(b, 15.0, 2e-3, 400, slab=0.8 * fovz)
            kz = ((il % 4) - 1.5) / fovz if k == 2 else (((il % 8) - 3.5) / fovz)
            blip = 100e-6
            b.add(np.full(10, blip / 10), gz=np.full(10, kz / (GAMMA * blip)))
            gx, gy = spiral_gradients(nro, 1e-6, nx / (2 * nx * d), 30e-3, rotation=il * np.pi / 2)
            b.add(np.full(nro, 1e-6), gx=gx, gy=gy, adc=np.ones(nro, bool))
            if k == 3:
                fill = 0.5 - (2e-3 + blip + nro * 1e-6)
                nfill = int(math.ceil(fill / 1e-3))
                b.add(np.full(nfill, fill / nfill))
        mask = "1111"
    else:
        raise ValueError("config index must be 0..3")

    def h_fn(t):
        h = field_waveforms(rng, t, amps)
        h[1] += np.asarray(b.gx)
        h[2] += np.asarray(b.gy)
        h[3] += np.asarray(b.gz)
        return h

    seq = b.build(h_fn)
    if spins_stride > 1:
        # A stride sharing a factor with a grid dimension would pick the same
        # few columns (e.g. only the masked-out edge): move to a coprime one.
        dims = {0: (64, 64), 1: (200, 200)}.get(k, (100, 100) if k == 2 else (200, 200))
        while any(math.gcd(spins_stride, d) != 1 for d in dims):
            spins_stride += 1
        sel = slice(0, None, spins_stride)
        x, y, z, rho, T1, T2, dw, csm = x[sel], y[sel], z[sel], rho[sel], T1[sel], T2[sel], dw[sel], csm[sel]
    obj = HO_Phantom(x=x, y=y, z=z, rho=rho, T1=T1, T2=T2, dw=dw, csm=csm, name=CONFIG_NAMES[k])
    parts, exc = get_sim_ranges(seq, max_block_length, max_block_length)
    state = Mag(np.zeros(len(obj), np.complex128), obj.rho.copy())
    return Workload(obj, seq, parts, exc, state, mask, CONFIG_NAMES[k])


@dataclass
class ServingRequest:
    obj: HO_Phantom
    seq: HO_DiscreteSequence
    parts: list
    excitation: list
    params: dict
    units: int  # spins x ADC samples x coils


def serving_request(rng) -> ServingRequest:
    """One request of the serving stream: spin count log-uniform in [1e3, 1e6]
    on a 2D or 3D grid over a 0.2 m FOV (ellipsoidal support), tissue as the
    2D single-coil configuration, a 90 degree hard pulse then a single-shot
    spiral of U[1k, 20k] ADC samples at 1-5 us dwell, 1/8/16/32 Gaussian
    coils, a random order mask, FP32 or FP64 arrays; every request runs on
    the split kernel (FP32 arrays are widened on the device and the results
    returned in FP32)."""
    ns_target = 10 ** rng.uniform(3.0, 6.0)
    fov = 0.2
    if rng.random() < 0.5:
        nx = ny = max(2, int(round(math.sqrt(ns_target))))
        nz = 1
    else:
        nz = max(2, int(round(ns_target ** (1.0 / 3.0) / 2)))
        nx = ny = max(2, int(round(math.sqrt(ns_target / nz))))
    d = fov / nx
    x, y, z = grid(nx, ny, nz, d, d, d)
    if nz == 1:
        z = np.zeros_like(x)
    rho, T1, T2, dw = tissue(rng, x.shape[0], 20.0)
    az = max(0.45 * nz * d, 1e-9)
    rho = rho * (((x / 0.09) ** 2 + (y / 0.09) ** 2 + (z / az) ** 2 if nz > 1 else (x / 0.09) ** 2 + (y / 0.09) ** 2)
                 <= 1.0)
    nc = int(rng.choice([1, 8, 16, 32]))
    if nc == 1:
        csm = np.ones((x.shape[0], 1), np.complex128)
    else:
        csm = gaussian_coils(rng, x, y, z, fibonacci_hemisphere(nc, 0.14), 0.08)
    nadc = int(rng.integers(1000, 20001))
    dwell = float(rng.integers(1, 6)) * 1e-6
    b = _SeqBuilder()
    b.hard_rf(90.0)
    gx, gy = spiral_gradients(nadc, dwell, nx / (2 * fov), 30e-3, rotation=rng.uniform(0, 2 * np.pi))
    b.add(np.full(nadc, dwell), gx=gx, gy=gy, adc=np.ones(nadc, bool))

    def h_fn(t):
        h = field_waveforms(rng, t, (1e-6, 1e-3, 5e-3, 20e-3))
        h[1] += np.asarray(b.gx)
        h[2] += np.asarray(b.gy)
        h[3] += np.asarray(b.gz)
        return h

    seq = b.build(h_fn)
    obj = HO_Phantom(x=x, y=y, z=z, rho=rho, T1=T1, T2=T2, dw=dw, csm=csm, name="serving")
    parts, exc = get_sim_ranges(seq, math.inf, math.inf)
    mask = format(int(rng.integers(0, 16)), "04b")
    f64 = bool(rng.random() < 0.5)
    if not f64:  # an FP32 caller holds FP32 arrays
        obj, seq = obj.astype(np.float32), seq.astype(np.float32)
    params = {"sim_method": BlochHighOrder(mask), "precision": "f64" if f64 else "f32",
              "homs_precision": "split"}
    return ServingRequest(obj, seq, parts, exc, params, x.shape[0] * nadc * nc)


def serving_pool(n: int, seed: int = 1004) -> List[ServingRequest]:
    """``n`` seeded requests of the serving stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [serving_request(rng) for _ in range(n)]


def _windowed_sinc_rf(b: _SeqBuilder, flip_deg, dur, nsteps, slab):
    """Hann-windowed sinc slab pulse (time-bandwidth 4) with slab-select Gz
    and a half-area rephasing lobe."""
    dt = dur / nsteps
    tc = (np.arange(nsteps) + 0.5) * dt - dur / 2
    tbw = 4.0
    bw = tbw / dur
    env = np.sinc(bw * tc) * (0.5 + 0.5 * np.cos(2 * np.pi * tc / dur))
    area = np.sum(env) * dt
    amp = (flip_deg / 360.0) / (GAMMA * area)
    b1 = amp * env
    gsel = bw / (GAMMA * slab)
    b.b1[-1] = b1[0]
    b1n = np.concatenate([b1[1:], [0.0]]).astype(np.complex128)
    b.add(np.full(nsteps, dt), gz=np.full(nsteps, gsel), b1=b1n, excitation=True)
    b.add(np.full(10, dur / 20), gz=np.full(10, -gsel))
