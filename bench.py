"""Benchmark: spin*sample*coil/s of the BlochHighOrder path on one B200 per rank.

Workload: the 3D 32-coil configuration (100x100x35 grid at 2 mm, 350,000
spins, 4 stack-of-spiral interleaves x 9,500 ADC samples at 1 us, full
third-order field waveforms, mask 1111), synthetic and seed-generated.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--mode split|plain]
    python bench.py --impl reference ...   # CPU oracle on the host cores

`value` is whole-job throughput with inputs resident on the device (a
prepared plan, signal written to device memory); `e2e` is the same metric
through the C ABI (homs_simulate) from pinned host buffers, with all
host<->device copies inside the timed region; `e2e_pipelined` is the same
again through the server (homs_server_submit, every step a request, two
slots), where one request's copies run beside another's kernels.  With N > 1
every rank runs an independent replica (the engine does not shard spins
across GPUs).

Further keys on one GPU: ``roofline`` (the algorithmic 8 flops per unit
against dense bf16), ``pipes`` (what the split kernel issues: int8 tensor
operations against the int8 rate, SFU operations against 16 per SM and clock
at the sampled clock), ``plain_f64`` (the plain FP64 kernel on the same
workload, device-timed, and the split/plain ratio), ``accuracy`` (signal
NRMSE of split and plain against the CPU FP64 oracle on a spin subsample, and
of split against plain FP64 at full size), ``configs`` (the 2D 1-coil, 2D
8-coil and 3D TR-loop workloads: split and plain throughput and NRMSE),
``cpu_baseline``, ``clocks``,
``serving`` / ``serving_resident`` (the mixed request stream),
``reference_gpu_equivalent`` (the reference's GPU design restated with
torch/cuBLAS and timed on the same workload), ``kspace`` (encoding export)
and ``phantom`` (device phantom builder).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "highordermrisim.jl_b200"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "spin*sample*coil/s"
UNIT = "spin*sample*coil/s"
CONFIG_INDEX = 2
FLOPS_PER_UNIT = 8.0  # one complex multiply-accumulate per spin*sample*coil
# What the split kernel issues per 32-spin x 128-sample chunk tile (N = 64 output columns):
# 3 phase MMAs of 128 x (160, 128, 64) x 32 int8 and 8 coil MMAs of 128 x (192, 192, 128, 64) x 32 int8
# (two K-steps of 16 spins).
I8_MACS_PER_SPIN_SAMPLE = (160 + 128 + 64 + 2 * (192 + 192 + 128 + 64)) * 32 / 32.0  # MACs per spin*sample
SFU_OPS_PER_SPIN_SAMPLE = 3.0  # sin, cos, ex2 on the MUFU (XU) pipe
SFU_PER_SM_CLK = 16.0  # MUFU results per SM and clock
# FP32 FMA-pipe operations the magnetisation warps write per spin*sample: the angle (1 FFMA), the decay
# argument (1), the top digits of Re/Im (2), their rounding residuals (2 FADD + 2 FFMA), the low digits (2).
FP32_OPS_PER_SPIN_SAMPLE = 10.0
FP32_PER_SM_CLK = 128.0  # FP32 lanes per SM and clock
FP64_FMA_PER_SM_CLK = 64.0  # FP64 FMA per SM and clock (37 TFLOP/s at 1,965 MHz)
N_SM = 148


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            p = json.load(fh)
        return float(p["bf16_tflops"]), float(p["hbm_gbs"]), "measured"
    except Exception:
        return 1590.0, 6650.0, "fallback"


def _traffic_per_launch():
    """DRAM bytes per launch of the split kernel, quoted from the committed ncu
    summary (not measured by this run: bench.py runs without a profiler)."""
    path = os.path.join(ROOT, "profiles", "split_precession_kernel_cfg2.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch_full:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, interval_ms: int = 50):
        self.device = device
        self.interval_ms = interval_ms
        self.proc = None
        self.lines = []
        self.first = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms",
                 str(self.interval_ms), "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def start_region(self, wait_s: float = 3.0):
        """Wait until nvidia-smi delivers samples, then count only later ones."""
        t0 = time.perf_counter()
        while self.proc is not None and not self.lines and time.perf_counter() - t0 < wait_s:
            time.sleep(0.01)
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        lines = self.lines[self.first:] or self.lines
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def replica_throughput(ms_local: float, units_per_rank: float, ws: int, device: str = "cuda"):
    """Whole-job throughput of N independent replicas: every rank processed
    `units_per_rank` in its own `ms_local`; the job's time is the slowest
    rank's (an all-reduce MAX over the process group when ws > 1).  Returns
    (units/s for all ranks together, max ms)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms_local)], dtype=torch.float64, device=device)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    return ws * units_per_rank / (ms_max / 1e3), ms_max


def _workload(stride=1, k=CONFIG_INDEX):
    from homs import workloads as W
    return W.config(k, spins_stride=stride)


def _workload_name(k, stride):
    from homs import workloads as W
    return W.CONFIG_NAMES[k] + (f"_every{stride}thspin" if stride > 1 else "")


def _units(w):
    from homs.model import count_block_adc
    return len(w.obj) * sum(count_block_adc(w.seq.adc, w.parts)) * w.obj.ncoils


def cpu_baseline(seconds_target=20.0, threads=None, k=CONFIG_INDEX, stride=None):
    """Time the CPU oracle (a port of the reference's CPU Float64 path) on a
    deterministic spin subsample of workload ``k``, on all host threads.

    The subsample is grown until one run takes about half of
    ``seconds_target`` (or taken as given by ``stride``).  Returns the
    baseline record, the stride, the subsampled workload and the oracle's
    signal: the same run is the checker of the GPU results on that subsample
    (``accuracy_on``)."""
    from homs.model import BlochHighOrder
    from oracle import oracle as orc
    orc.build()
    if threads is None:
        threads = max(1, len(os.sched_getaffinity(0)))
    fixed = stride is not None
    stride = stride or 400
    while True:
        w = _workload(stride=stride, k=k)
        flags = BlochHighOrder(w.mask).flags
        t0 = time.perf_counter()
        sig = orc.simulate_c(w.obj, w.seq, w.parts, w.excitation, flags, nthreads=threads)[0]
        dt = time.perf_counter() - t0
        if fixed or dt >= seconds_target / 2 or stride == 1:
            break
        # The oracle's cost per spin grows with the sample (cache), so a prediction from a small sample
        # overshoots: aim at half the target and take at most 16x more spins per step.
        stride = max(1, int(2.0 * stride * dt / seconds_target), stride // 16)
    from homs.model import count_block_adc
    nadc = sum(count_block_adc(w.seq.adc, w.parts))
    return ({"value": _units(w) / dt, "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": _cpu_model(),
             "affinity_cpus": len(os.sched_getaffinity(0)),
             "sample": f"every {stride}th spin ({len(w.obj)} spins) x {nadc} samples x {w.obj.ncoils} coils, full "
                       f"sequence, {dt:.2f} s"}, stride, w, sig)


def accuracy_on(w, ref_sig, ctx, modes=("split", "plain")):
    """Signal NRMSE of the engine's modes against the oracle signal of the
    same (subsampled) workload, both from FP64 arrays."""
    import homs
    from homs.model import BlochHighOrder
    method = BlochHighOrder(w.mask)
    den = float(np.linalg.norm(ref_sig))
    out = {}
    for mode in modes:
        got = homs.run_blocks(w.obj, w.seq, w.parts, w.excitation, method, "f64", mode, context=ctx)[0]
        out[mode] = float(np.linalg.norm(got - ref_sig) / den)
    return out


def time_plan(ctx, w, mode, precision="f64", steps=3, warmup=1):
    """Device time of prepared-plan runs of workload ``w`` (inputs resident,
    signal to device memory; CUDA events on the context's stream).  Returns
    the timing record and the last run's signal (device tensor, Nc x Nadc)."""
    import torch

    import homs
    from homs import _lib
    from homs.model import BlochHighOrder
    lib = _lib.load()
    params = {"sim_method": BlochHighOrder(w.mask), "precision": precision, "homs_precision": mode}
    plan = homs.prepare_simulation(w.obj, w.seq, sim_params=params, parts=w.parts, excitation=w.excitation,
                                   context=ctx)
    sig = torch.empty((plan.nc, plan.nadc), dtype=torch.complex128 if precision == "f64" else torch.complex64,
                      device="cuda")

    def step():
        _lib.check(lib.homs_plan_run(plan.handle, ctypes.c_void_p(sig.data_ptr()), _lib.HOMS_DEVICE, None),
                   ctx.handle)

    for _ in range(warmup):
        step()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    fused_ms, fused_n = 0.0, 0
    a.record(stream)
    for _ in range(steps):
        step()
        t = _lib.Timing()
        _lib.check(lib.homs_plan_timing(plan.handle, ctypes.byref(t)))
        fused_ms += t.fused_kernel_ms
        fused_n += t.fused_launches
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    plan.close()
    units = _units(w)
    return {"ms_per_step": ms, "units_per_s": units / (ms / 1e3), "steps": steps, "warmup": warmup,
            "fused_kernel_ms_per_launch": fused_ms / max(fused_n, 1)}, sig


def config_legs(ctx):
    """The other named workloads: split and plain FP64 throughput (device
    time of plan runs) and each mode's signal NRMSE against the CPU oracle
    on a spin subsample (the oracle run is that config's CPU baseline).  The
    3D TR loop runs split at full size and plain FP64 on every 20th spin
    (its time is linear in the spin count; 32 s per full step)."""
    import torch
    out = {}
    for k, split_stride, plain_stride, oracle_stride, steps in ((0, 1, 1, 1, 5), (1, 1, 1, 1, 3),
                                                                (3, 1, 20, 2003, 1)):
        from homs import workloads as W
        rec = {"workload": _workload_name(k, 1)}
        w = _workload(split_stride, k)
        sp, _ = time_plan(ctx, w, "split", steps=steps, warmup=1)
        rec["split"] = dict(sp, spins=len(w.obj))
        wp = w if plain_stride == split_stride else _workload(plain_stride, k)
        pl, _ = time_plan(ctx, wp, "plain", steps=1 if k == 3 else steps, warmup=1)
        rec["plain_f64"] = dict(pl, spins=len(wp.obj), sample=(f"every {plain_stride}th spin" if plain_stride > 1
                                                                  else "full workload"))
        rec["split_over_plain_f64"] = sp["units_per_s"] / pl["units_per_s"]
        del w, wp
        torch.cuda.empty_cache()
        base, stride, ws, ref = cpu_baseline(k=k, stride=oracle_stride)
        rec["cpu_baseline"] = base
        rec["nrmse_vs_oracle"] = dict(accuracy_on(ws, ref, ctx), sample=base["sample"])
        out[W.CONFIG_NAMES[k]] = rec
    return out


def serving_benchmark(n_pool=16, passes=20, load=0.95, slots=4, resident=False, spin_sample_rate=None):
    """Serving stream of mixed simulations through homs.Server.

    Batch mode submits every request at once (the server's capacity);
    serving mode submits the same requests with Poisson arrivals at ``load``
    times the batch request rate.  Latency is finish - submit per request;
    sustained throughput is total units over first submit to last finish.
    With ``resident`` every distinct phantom is put on the device once, before
    the timed streams (homs.ResidentPhantom), and requests carry only their
    sequences; otherwise every request uploads its phantom.

    ``spin_sample_rate`` (the headline kernel's spin*sample/s) gives the mix's
    kernel bound: units count coils, so a mix of 1- to 32-coil requests
    reaches at most that rate times its spin*sample-weighted coil count."""
    import homs
    from homs import workloads as W
    pool = W.serving_pool(n_pool)
    reqs = [pool[i % n_pool] for i in range(n_pool * passes)]
    units = float(sum(r.units for r in reqs))
    spin_samples = float(sum(len(r.obj) * int(np.count_nonzero(np.asarray(r.seq.adc))) for r in reqs))
    residents = {}
    if resident:
        for r in pool:
            residents[id(r)] = homs.ResidentPhantom(r.obj, r.params["precision"], r.params["homs_precision"])

    def submit(srv, r):
        obj = residents.get(id(r), r.obj)
        return srv.submit(obj, r.seq, sim_params=r.params, parts=r.parts, excitation=r.excitation)

    with homs.Server(slots=slots) as srv:
        # Warm-up: the whole batch once, so that every slot's device workspace
        # has grown to the requests it may get (a growth frees device memory,
        # which waits for the whole device) before anything is timed.
        for t in [submit(srv, r) for r in reqs]:
            srv.result(t)
            srv.release(t)
        t0 = time.perf_counter()
        tickets = [submit(srv, r) for r in reqs]
        for t in tickets:
            srv.result(t)
        batch_s = time.perf_counter() - t0
        for t in tickets:
            srv.release(t)
        rate = len(reqs) / batch_s * load
        rng = np.random.default_rng(7)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
        tickets = []
        t0 = time.perf_counter()
        for r, at in zip(reqs, arrivals):
            wait = at - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            tickets.append(submit(srv, r))
        for t in tickets:
            srv.result(t)
        spans = [srv.times(t) for t in tickets]
    for res in residents.values():
        res.close()
    lat = np.array([f - s for s, _, f in spans]) * 1e3
    makespan = max(f for _, _, f in spans) - min(s for s, _, _ in spans)
    sustained = units / makespan
    # What the arrivals offered: units over first to last submit.  A server that
    # keeps up finishes the stream one request latency after the last arrival.
    offered = units / (max(s for s, _, _ in spans) - min(s for s, _, _ in spans))
    batch = units / batch_s
    bound = {}
    if spin_sample_rate:
        kb = spin_sample_rate * units / spin_samples
        bound = {"mix_coils_per_spin_sample": units / spin_samples, "kernel_bound_units_per_s": kb,
                 "batch_fraction_of_kernel_bound": batch / kb,
                 "kernel_bound": "the headline split kernel's spin*sample rate x the mix's spin*sample-weighted "
                                 "coil count"}
    return {"requests": len(reqs), "distinct": n_pool, "slots": slots, "load": load,
            "arrival_rate_per_s": rate, "batch_units_per_s": batch, "sustained_units_per_s": sustained,
            **bound,
            "fraction_of_batch": sustained / batch, "offered_units_per_s": offered,
            "sustained_over_offered": sustained / offered, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat.max()),
            "mix": "spins log-uniform 1e3-1e6, 2D/3D, ADC U[1k,20k] at 1-5 us, coils {1,8,16,32}, random masks, "
                   "f32 or f64 arrays, all on the split kernel (the server's rounds: one persistent launch per "
                   "output width over all requests' current segments)",
            "phantoms": "resident on the device (uploaded once, before the streams)" if resident else
                        "uploaded from pageable host memory by every request (staged through page-locked "
                        "chunks)"}


def plain_per_request(n_pool=16):
    """The plain per-request kernel: every distinct request of the serving
    pool once, one at a time, on the reference-order plain kernel in its own
    precision (phantom uploaded per request)."""
    import homs
    from homs import workloads as W
    pool = W.serving_pool(n_pool)
    units, secs = 0.0, 0.0
    for r in pool:
        params = dict(r.params, homs_precision="plain")
        t0 = time.perf_counter()
        homs.simulate(r.obj, r.seq, sim_params=params, parts=r.parts, excitation=r.excitation)
        secs += time.perf_counter() - t0
        units += r.units
    return units / secs


def kspace_benchmark(ctx, hbm_peak, peak_kind, reps=20):
    """Encoding export (homs_kspace) on the 3D TR-loop sequence: 364,316
    nodes, 35 excitation breaks, 19 columns (gx, gy, gz, h0..h15) and the
    332,500 ADC times.  Kernel time from the CUDA events libhoms records
    around its four kernels; end to end is the host call (pageable copies of
    the 21 sequence arrays in, k and k at the ADC times out); the NumPy
    restatement of grad2kspace is timed beside it on one host thread."""
    import ctypes as ct
    import homs
    from homs import _lib
    from homs import workloads as W
    from oracle import oracle as orc
    seq = W.config(3, spins_stride=20001).seq
    starts, signs = homs.rf_events(seq)
    q = np.asarray(seq.t)[np.asarray(seq.adc)]
    nn, nq = seq.nnodes, q.shape[0]
    m = nn - 1
    lib = _lib.load()
    kernel_ms, wall_ms = [], []
    for i in range(reps + 3):
        t0 = time.perf_counter()
        homs.get_kspace(seq, rf_start=starts, rf_sign=signs, adc_times=q, context=ctx)
        wall = (time.perf_counter() - t0) * 1e3
        d = ct.c_double()
        _lib.check(lib.homs_kspace_timing(ctx.handle, ct.byref(d)), ctx.handle)
        if i >= 3:
            kernel_ms.append(d.value)
            wall_ms.append(wall)
    t0 = time.perf_counter()
    orc.grad2kspace_np(seq, starts, signs, homs.GAMMA, q)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    alg_bytes = 8 * (19 * nn + m + 19 * m + 19 * nq)  # 19 columns and dt in; k and k at the ADC times out
    dev_ms = statistics.median(kernel_ms)
    achieved = alg_bytes / (dev_ms / 1e3) / 1e9
    return {"workload": f"3D TR-loop sequence: {nn} nodes, {len(starts)} RF breaks, 19 columns, {nq} ADC times",
            "kernel_ms": dev_ms, "algorithmic_bytes": alg_bytes,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "peak_source": f"{peak_kind} HBM copy (MEASURED_PEAKS.json)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s"},
            "e2e_ms": statistics.median(wall_ms), "kernels_per_call": 4,
            "l2": "inputs (55 MB) smaller than L2; copied in by the call itself",
            "cpu_oracle_ms": cpu_ms, "cpu_oracle": "NumPy restatement of grad2kspace, 1 thread"}


def phantom_benchmark(ctx, hbm_peak, peak_kind, reps=5):
    """Brain phantom builder (homs_brain_phantom_fill) on a 200 x 200 x 50
    class volume (2,000,000 voxels, seeded classes of the brain phantom with
    background) with a 32-coil receive map, device memory in and out.  Times
    the fill call (its count pass, the offsets scan and the compaction) with
    CUDA events on the context's stream; the NumPy restatement is timed on
    the host beside it."""
    import ctypes as ct
    import torch
    from homs import _lib
    from oracle import oracle as orc
    rng = np.random.default_rng(1005)
    shape, nc = (200, 200, 50), 32
    classes = np.array([23, 46, 70, 93, 116, 139, 162, 185, 209, 232, 255, 0, 0, 0], np.uint8)
    lab = rng.choice(classes, size=shape)
    nvox = lab.size
    lab_d = torch.as_tensor(np.asfortranarray(lab).ravel(order="F"), device="cuda")
    csm_d = torch.randn(nvox * nc, dtype=torch.complex128, device="cuda")
    spec = _lib.BrainSpec()
    spec.nx, spec.ny, spec.nz = shape
    spec.res[:] = [1e-3] * 3
    spec.offcenter[:] = [0.0] * 3
    spec.fieldstrength, spec.ncoils, spec.memory = 0, nc, _lib.HOMS_DEVICE
    spec.labels, spec.fieldmap, spec.csm = lab_d.data_ptr(), None, csm_d.data_ptr()
    lib = _lib.load()
    n = ct.c_int64()
    _lib.check(lib.homs_brain_phantom_count(ctx.handle, ct.byref(spec), ct.byref(n)), ctx.handle)
    ns = int(n.value)
    outs = [torch.empty(ns, dtype=torch.float64, device="cuda") for _ in range(8)]
    csm_o = torch.empty(ns * nc, dtype=torch.complex128, device="cuda")
    out = _lib.BrainOut()
    out.nspins, out.memory = ns, _lib.HOMS_DEVICE
    for k, t in zip(("x", "y", "z", "rho", "T1", "T2", "T2s", "dw"), outs):
        setattr(out, k, t.data_ptr())
    out.csm = csm_o.data_ptr()
    stream = torch.cuda.current_stream()
    times = []
    for i in range(reps + 2):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        _lib.check(lib.homs_brain_phantom_fill(ctx.handle, ct.byref(spec), ct.byref(out)), ctx.handle)
        b.record(stream)
        torch.cuda.synchronize()
        if i >= 2:
            times.append(a.elapsed_time(b))
    ms = statistics.median(times)
    # labels read twice (count and fill) and the map once; 8 spin arrays and the compacted map written
    alg = 2 * nvox + 16 * nvox * nc + 8 * 8 * ns + 16 * ns * nc
    t0 = time.perf_counter()
    orc.brain_phantom_np(lab, (1e-3,) * 3, csm=None)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    achieved = alg / (ms / 1e3) / 1e9
    return {"workload": f"brain class volume 200x200x50 ({nvox} voxels, {ns} spins kept), 32-coil map, device in/out",
            "ms": ms, "algorithmic_bytes": alg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "peak_source": f"{peak_kind} HBM copy (MEASURED_PEAKS.json)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s"},
            "cpu_oracle_ms_unit_coil": cpu_ms,
            "timing": "CUDA events on the context's stream around the call (count pass, scan, compaction)"}


def coil_reduce_benchmark(hbm_peak, peak_kind, ns=200000, nadc=64, nc=32, reps=20):
    """Standalone coil reduction (homs_coil_reduce, the reference's
    CoilReductionGPU entry, kernels/CoilReductionGPU.jl:79-100,212-233):
    signal = states^T csm for 200,000 spins x 64 ADC states x 32 coils, FP64,
    device memory in and out.  Times the call (the reduction over spin tiles
    and the fixed-order sum of the tile partials) with CUDA events on the
    context's stream."""
    import ctypes as ct
    import torch
    from homs import _lib
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(1006)
    states = torch.randn((nadc, ns), dtype=torch.complex128, device="cuda", generator=g)  # ns x nadc, column-major
    csm = torch.randn((nc, ns), dtype=torch.complex128, device="cuda", generator=g)  # ns x nc, column-major
    sig = torch.empty((nc, nadc), dtype=torch.complex128, device="cuda")
    # A context on an explicit stream, so that the events bracket the call's kernels.
    stream = torch.cuda.Stream()
    times = []
    with _lib.Context(torch.cuda.current_device(), stream.cuda_stream) as rctx:
        for i in range(reps + 3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            _lib.check(lib.homs_coil_reduce(rctx.handle, _lib.HOMS_F64, ns, nadc, nc, ct.c_void_p(states.data_ptr()),
                                            ns, ct.c_void_p(csm.data_ptr()), ns, ct.c_void_p(sig.data_ptr()), nadc),
                       rctx.handle)
            b.record(stream)
            torch.cuda.synchronize()
            if i >= 3:
                times.append(a.elapsed_time(b))
    ref = states @ csm.T  # (nadc x nc): sum over spins of state x sensitivity, no conjugation
    err = float(torch.linalg.norm(sig.T - ref) / torch.linalg.norm(ref))
    ms = statistics.median(times)
    tiles = -(-ns // 256)
    # states and sensitivities read once, the signal written; the tile partials
    # (written and read back once) are the deterministic reduction's own traffic
    alg = 16 * (ns * nadc + ns * nc + nadc * nc)
    partial_bytes = 2 * 16 * tiles * nadc * nc
    achieved = alg / (ms / 1e3) / 1e9
    return {"workload": f"{ns} spins x {nadc} states x {nc} coils, FP64, device in/out",
            "ms": ms, "algorithmic_bytes": alg, "partial_bytes": partial_bytes,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "peak_source": f"{peak_kind} HBM copy (MEASURED_PEAKS.json)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s"},
            "nrmse_vs_torch_f64": err,
            "timing": "CUDA events on the context's stream around the call (reduction and partial sum)"}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from homs.model import BlochHighOrder
    from oracle import oracle as orc
    # Calibrate a spin subsample of a few seconds per step, then time each
    # step on that same subsample and report what was timed; the projection
    # to the full workload (the oracle's time is linear in the spin count)
    # is a separate, labelled field.
    base, stride, w, _ = cpu_baseline(seconds_target=max(3.0, 30.0 / max(args.steps + args.warmup, 1)))
    flags = BlochHighOrder(w.mask).flags
    threads = base["cores"]
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        orc.simulate_c(w.obj, w.seq, w.parts, w.excitation, flags, nthreads=threads)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    step_s = statistics.median(times)
    units = _units(w)
    v = units / step_s
    full = _workload(1)
    full_units = _units(full)
    nadc = units // (len(w.obj) * w.obj.ncoils)
    base["value"] = v
    base["sample"] = (f"every {stride}th spin ({len(w.obj)} spins) x {nadc} samples x {w.obj.ncoils} coils per "
                      f"step, median of {args.steps} steps")
    base["projection"] = {"workload": _workload_name(CONFIG_INDEX, 1), "spins": len(full.obj),
                          "ms_per_step": full_units / v * 1e3, "extrapolated": True,
                          "basis": "the oracle's cost is linear in the spin count"}
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": step_s * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": _workload_name(CONFIG_INDEX, stride), "spins": len(w.obj),
                      "spins_timed": len(w.obj), "stride": stride, "samples": int(nadc), "coils": w.obj.ncoils,
                      "mask": w.mask, "extrapolated": False},
           "impl": "reference", "cpu_baseline": base,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def run_homs(args):
    import torch
    import torch.distributed as dist

    import homs
    from homs import _lib
    from homs.model import BlochHighOrder

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    stream = torch.cuda.current_stream()
    ctx = _lib.Context(local, stream.cuda_stream)
    lib = _lib.load()
    w = _workload(args.spin_stride, args.config)
    units = _units(w)
    method = BlochHighOrder(w.mask)
    params = {"sim_method": method, "precision": args.precision, "homs_precision": args.mode}
    plan = homs.prepare_simulation(w.obj, w.seq, sim_params=params, parts=w.parts, excitation=w.excitation,
                                   context=ctx)
    nadc, nc = plan.nadc, plan.nc
    sig_dev = torch.empty((nc, nadc), dtype=torch.complex128 if args.precision == "f64" else torch.complex64,
                          device="cuda")

    def device_step():
        _lib.check(lib.homs_plan_run(plan.handle, ctypes.c_void_p(sig_dev.data_ptr()), _lib.HOMS_DEVICE, None),
                   ctx.handle)

    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        device_step()
    barrier()
    fused_ms, fused_n, launches = 0.0, 0, 0
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        clocks.start_region()
        start.record(stream)
        for _ in range(args.steps):
            device_step()
            t = _lib.Timing()
            _lib.check(lib.homs_plan_timing(plan.handle, ctypes.byref(t)))
            fused_ms += t.fused_kernel_ms
            fused_n += t.fused_launches
            launches += t.kernel_launches
        stop.record(stream)
        barrier()
    ms = start.elapsed_time(stop) / args.steps
    value, ms_max = replica_throughput(ms, units, ws)
    plan.close()

    # End to end through the C ABI from pinned host memory.
    e2e = e2e_pipelined = None
    if not args.no_e2e:
        keep = _lib._Keep()
        pin = lambda a: _pinned(torch, a)  # noqa: E731
        obj, seq = w.obj, w.seq
        rt = np.float64 if args.precision == "f64" else np.float32
        ct = np.complex128 if args.precision == "f64" else np.complex64
        dcode = _lib.HOMS_F64 if args.precision == "f64" else _lib.HOMS_F32
        ph = _lib.Phantom(len(obj), nc, dcode, _lib.HOMS_HOST,
                          *[keep.ptr(pin(np.asarray(v, rt))) for v in
                            (obj.x, obj.y, obj.z, obj.rho, obj.T1, obj.T2, obj.dw)],
                          keep.ptr(pin(np.asfortranarray(obj.csm.astype(ct)))))
        hp = [pin(np.ascontiguousarray(seq.h[k], rt)) for k in range(16)]
        keep.items.extend(hp)
        first = np.array([p[0] for p in w.parts], np.int64)
        last = np.array([p[1] for p in w.parts], np.int64)
        exc = np.array(w.excitation, np.uint8)
        sq = _lib.Sequence(len(seq.t), dcode, _lib.HOMS_HOST,
                           *[keep.ptr(pin(np.asarray(v, rt))) for v in (seq.t, seq.dt, seq.gx, seq.gy, seq.gz)],
                           keep.ptr(pin(np.asarray(seq.b1, ct))), keep.ptr(pin(np.asarray(seq.df, rt))),
                           keep.ptr(pin(np.asarray(seq.psi, rt))),
                           keep.ptr(pin(np.asarray(seq.adc, np.uint8))),
                           (ctypes.c_void_p * 16)(*[a.ctypes.data for a in hp]), len(w.parts), keep.ptr(first),
                           keep.ptr(last), keep.ptr(exc), homs.GAMMA)
        sig_h = pin(np.zeros((nc, nadc), ct))
        xy_h = pin(np.zeros(len(obj), ct))
        z_h = pin(np.asarray(obj.rho, rt).copy())
        st = _lib.State(xy_h.ctypes.data, z_h.ctypes.data, _lib.HOMS_HOST)
        opts = _lib.RunOptions()
        opts.method = method.flags
        opts.mode = _lib.HOMS_SPLIT if args.mode == "split" else _lib.HOMS_PLAIN
        h2d = sum(a.nbytes for a in keep.items if isinstance(a, np.ndarray)) + xy_h.nbytes + z_h.nbytes
        d2h = sig_h.nbytes + xy_h.nbytes + z_h.nbytes

        def e2e_step():
            xy_h[:] = 0
            z_h[:] = obj.rho
            _lib.check(lib.homs_simulate(ctx.handle, ctypes.byref(ph), ctypes.byref(sq), ctypes.byref(opts),
                                         ctypes.byref(st), sig_h.ctypes.data, _lib.HOMS_HOST), ctx.handle)

        for _ in range(args.warmup):
            e2e_step()
        barrier()
        t0 = time.perf_counter()
        n_e2e = args.steps
        for _ in range(n_e2e):
            e2e_step()
        barrier()
        e_ms = (time.perf_counter() - t0) * 1e3 / n_e2e
        e_value, e_max = replica_throughput(e_ms, units, ws)
        e2e = {"value": e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e_max, "steps": n_e2e, "warmup": args.warmup,
               "timing": "host wall time of homs_simulate calls (pinned host buffers, copies inside)"}

        # The same simulations through the server (homs_server_submit): all
        # requests submitted at once to 2 slots, each with its own page-locked
        # state and signal, so that one request's copies and operand builds run
        # beside another's kernels.  Copies stay inside the timed region.
        sopt = _lib.ServerOptions()
        sopt.device = torch.cuda.current_device()
        sopt.slots = 2
        srv = ctypes.c_void_p()
        _lib.check(lib.homs_server_create(ctypes.byref(sopt), ctypes.byref(srv)))
        try:
            def pipelined(n):
                bufs = [(pin(np.zeros((nc, nadc), ct)), pin(np.zeros(len(obj), ct)),
                         pin(np.asarray(obj.rho, rt).copy())) for _ in range(n)]
                sts = [_lib.State(b[1].ctypes.data, b[2].ctypes.data, _lib.HOMS_HOST) for b in bufs]
                barrier()
                t0 = time.perf_counter()
                tickets = []
                for b, s in zip(bufs, sts):
                    t = ctypes.c_int64()
                    _lib.check(lib.homs_server_submit(srv, ctypes.byref(ph), ctypes.byref(sq), ctypes.byref(opts),
                                                      ctypes.byref(s), b[0].ctypes.data, _lib.HOMS_HOST,
                                                      ctypes.byref(t)))
                    tickets.append(t.value)
                for t in tickets:
                    st_ = lib.homs_server_wait(srv, t, 600.0)
                    if st_ != 0:
                        raise RuntimeError((lib.homs_server_error(srv, t) or b"").decode())
                dt_ = time.perf_counter() - t0
                barrier()
                for t in tickets:
                    lib.homs_server_release(srv, t)
                return dt_

            pipelined(2)  # warm-up: both slots' workspaces grow
            n_p = max(args.steps, 4)
            p_ms = pipelined(n_p) * 1e3 / n_p
            p_value, p_max = replica_throughput(p_ms, units, ws)
            e2e_pipelined = {"value": p_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                             "d2h_bytes_per_step": int(d2h), "ms_per_step": p_max, "requests": n_p, "slots": 2,
                             "timing": "host wall time from the first homs_server_submit to the last completion "
                                       "(pinned host buffers, copies inside)"}
        finally:
            lib.homs_server_destroy(srv)

    if rank != 0:
        if ws > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    bf16_peak, hbm_peak, peak_kind = _peaks()
    seg_units = units * args.steps / max(fused_n, 1)  # units per fused launch
    avg_launch_ms = fused_ms / max(fused_n, 1)
    achieved_tflops = FLOPS_PER_UNIT * seg_units / (avg_launch_ms / 1e3) / 1e12 if avg_launch_ms > 0 else None
    traffic = _traffic_per_launch() if (args.config == CONFIG_INDEX and args.mode == "split"
                                        and args.spin_stride == 1) else None
    roof = {"bound": "tensor", "achieved": achieved_tflops, "peak": bf16_peak, "unit": "TFLOP/s",
            "frac": (achieved_tflops / bf16_peak) if achieved_tflops else None, "traffic": traffic,
            "peak_source": f"{peak_kind} dense bf16 (MEASURED_PEAKS.json)" if peak_kind == "measured" else
            "fallback 1.59 PFLOP/s", "kernel": "split_precession_kernel" if args.mode == "split" else
            "segment_kernel", "kernel_ms_per_launch": avg_launch_ms,
            "units_per_launch": seg_units, "flops_per_unit": FLOPS_PER_UNIT}
    if traffic is not None:
        roof["traffic_source"] = "quoted from profiles/split_precession_kernel_cfg2.md (one ncu capture)"
    clk = clocks.summary()
    pipes = None
    if args.mode == "split" and avg_launch_ms > 0:
        # What the split kernel issues, from the same launch times: int8 tensor MACs (exact digit
        # products) against the int8 rate (twice the dense bf16 rate per MMA shape on sm_100: the
        # measured bf16 peak x 2; 4.5 POPS nominal) and MUFU ops (sin, cos, ex2) against 16 per SM and
        # clock at the median sampled SM clock.
        secs = avg_launch_ms / 1e3
        spin_samples = seg_units / nc
        i8_tops = 2.0 * I8_MACS_PER_SPIN_SAMPLE * spin_samples / secs / 1e12
        mhz = clk.get("sm_mhz") or 1965.0
        sfu_peak = SFU_PER_SM_CLK * N_SM * mhz * 1e6
        pipes = {"int8_tensor_tops": i8_tops, "int8_macs_per_spin_sample": I8_MACS_PER_SPIN_SAMPLE,
                 "int8_peak_tops": 2.0 * bf16_peak, "int8_frac": i8_tops / (2.0 * bf16_peak),
                 "int8_peak_source": f"2 x {peak_kind} dense bf16",
                 "sfu_ops_per_s": SFU_OPS_PER_SPIN_SAMPLE * spin_samples / secs,
                 "sfu_ops_per_spin_sample": SFU_OPS_PER_SPIN_SAMPLE, "sfu_peak_ops_per_s": sfu_peak,
                 "sfu_frac": SFU_OPS_PER_SPIN_SAMPLE * spin_samples / secs / sfu_peak,
                 "sfu_peak_source": f"{SFU_PER_SM_CLK:.0f} per SM and clock x {N_SM} SMs x {mhz:.0f} MHz (sampled)",
                 "fp32_ops_per_spin_sample": FP32_OPS_PER_SPIN_SAMPLE,
                 "fp32_frac": FP32_OPS_PER_SPIN_SAMPLE * spin_samples / secs / (FP32_PER_SM_CLK * N_SM * mhz * 1e6),
                 "fp32_peak_source": f"{FP32_PER_SM_CLK:.0f} lanes per SM and clock x {N_SM} SMs x {mhz:.0f} MHz "
                                     "(sampled); the ops are those the kernel's source writes",
                 "spin_samples_per_launch": spin_samples, "kernel_ms_per_launch": avg_launch_ms}
    base = accuracy = None
    if ws == 1 and not args.no_cpu_baseline:
        base, _, w_sub, ref_sub = cpu_baseline(k=args.config)
        accuracy = {"sample": base["sample"], "nrmse_vs_oracle": accuracy_on(w_sub, ref_sub, ctx)}
        del w_sub, ref_sub
    plain = None
    if ws == 1 and args.mode == "split" and not args.no_plain:
        pl, sig_plain = time_plan(ctx, w, "plain", precision=args.precision, steps=3, warmup=1)
        mhz = clk.get("sm_mhz") or 1965.0
        fp64_peak = 2.0 * FP64_FMA_PER_SM_CLK * N_SM * mhz * 1e6
        plain = dict(pl, split_over_plain_f64=value / pl["units_per_s"],
                     coil_fp64_flops_per_s=FLOPS_PER_UNIT * pl["units_per_s"],
                     coil_fp64_frac=FLOPS_PER_UNIT * pl["units_per_s"] / fp64_peak,
                     fp64_peak_source=f"{FP64_FMA_PER_SM_CLK:.0f} FMA per SM and clock x {N_SM} SMs x {mhz:.0f} MHz "
                                      "(sampled; FP64 is not among the measured peaks); counts only the coil "
                                      "contraction's 8 flops per unit, not the field, phase and sincos/exp",
                     note="the plain kernel (the reference's per-spin sequential trapezoid, FP64) on the same "
                          "workload, device-timed plan runs")
        d = float(torch.linalg.vector_norm(sig_plain).item())
        nr = float(torch.linalg.vector_norm(sig_dev - sig_plain).item()) / d
        if accuracy is None:
            accuracy = {}
        accuracy["nrmse_split_vs_plain_f64_full"] = nr
        del sig_plain
        torch.cuda.empty_cache()
    nchunks = -(-len(w.obj) // 32)
    ncg = min(nc, 32)
    n_cols = max(16, -(-2 * ncg // 16) * 16)
    # phase digits (11,264 B per 32-spin chunk) and the sensitivity digits per coil group
    op_mb = nchunks * (11264 + 6 * n_cols * 32 * -(-nc // 32)) / 1e6 if args.mode == "split" else 0.0
    csm_mb = len(w.obj) * nc * 16 / 1e6
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": ("int8 tensor: fixed-point phase (5 digits) and coil contraction (3 digits), exact int32 sums;"
                     " f32 sfu trig; f64 tables") if args.mode == "split" else args.precision,
           "data": "synthetic",
           "config": {"workload": _workload_name(args.config, args.spin_stride), "spins": len(w.obj),
                      "samples": nadc, "coils": nc, "mask": w.mask, "mode": args.mode,
                      "l2": (f"inputs larger than L2 (csm {csm_mb:.0f} MB" +
                             (f", split operand {op_mb:.0f} MB)" if op_mb else ")")) if csm_mb > 126 else
                      f"inputs smaller than L2 (csm {csm_mb:.0f} MB)", "parallelism": f"replicas{ws}"},
           "roofline": roof, "pipes": pipes, "plain_f64": plain, "accuracy": accuracy, "cpu_baseline": base,
           "e2e": e2e, "e2e_pipelined": e2e_pipelined, "gpu_launches": launches, "clocks": clk}
    if ws == 1 and not args.no_configs and args.config == CONFIG_INDEX and args.spin_stride == 1:
        out["configs"] = config_legs(ctx)
    if ws == 1 and not args.no_serve:
        ss_rate = value / nc if args.mode == "split" and args.spin_stride == 1 else None
        out["serving"] = serving_benchmark(spin_sample_rate=ss_rate)
        out["serving"]["plain_per_request_units_per_s"] = plain_per_request()
        out["serving_resident"] = serving_benchmark(resident=True, spin_sample_rate=ss_rate)
    if ws == 1 and not args.no_refgpu and args.config == CONFIG_INDEX and args.spin_stride == 1:
        out["reference_gpu_equivalent"] = reference_gpu_leg(w, sig_dev, ms_max, units)
    if ws == 1 and not args.no_kspace:
        out["kspace"] = kspace_benchmark(ctx, hbm_peak, peak_kind)
        out["phantom"] = phantom_benchmark(ctx, hbm_peak, peak_kind)
        out["coil_reduce"] = coil_reduce_benchmark(hbm_peak, peak_kind)
    print(json.dumps(out))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def reference_gpu_equivalent(w, dtype: str = "f32", block: int = 32, device: str = "cuda", time_it: bool = True,
                             graph: bool = False, times: dict = None):
    """The reference's own GPU design, restated with torch and cuBLAS and run on
    this GPU: the comparator for the fused kernels (not part of the product).

    Excitation parts step an elementwise spinor over the spins per node
    (kernels/HighOrderGPU.jl:181-233).  Precession runs in blocks of at most
    ``block`` intervals, as the reference's workspace is sized
    (kernels/HighOrderGPU.jl:6-58): per block, the field of every spin and node
    is a (spins x 17) by (17 x nodes) GEMM of the unnormalised basis against the
    masked coefficients (:63-93), the phase its trapezoid sum, and the states
    M0 exp(i phi - t/T2) at the block's ADC nodes are materialised and reduced
    into the coils by one complex GEMM, states^T csm (:95-178, the default
    "gemm" coil combination).  The state carries across blocks and parts.

    With ``graph`` the whole run is captured once into a CUDA graph and the
    timed run is its replay, so the host loop's launch overhead is excluded;
    ``times`` (a dict) then receives ``eager_ms`` (the host loop) and
    ``graph_ms`` (the replay).

    Returns (signal (Nadc x Nc) as numpy, ms on the device or None)."""
    import torch

    from homs.model import GAMMA, BlochHighOrder
    rt = torch.float64 if dtype == "f64" else torch.float32
    ct = torch.complex128 if dtype == "f64" else torch.complex64
    dev = torch.device(device)
    obj, seq = w.obj, w.seq
    T = lambda a, d=rt: torch.as_tensor(np.ascontiguousarray(a), device=dev).to(d)  # noqa: E731
    x, y, z, rho, T1, T2, dw = (T(getattr(obj, k)) for k in ("x", "y", "z", "rho", "T1", "T2", "dw"))
    csm = T(np.asarray(obj.csm), ct)
    m = BlochHighOrder(w.mask).flags
    ho0, ho1, ho2, ho3, dw_exc, dw_prec = (bool(m & b) for b in (1, 2, 4, 8, 16, 32))
    r2 = x * x + y * y + z * z
    one = torch.ones_like(x)
    basis = torch.stack([one, x, y, z, x * y, z * y, 3 * z * z - r2, x * z, x * x - y * y,
                         3 * y * x * x - y ** 3, x * z * y, (5 * z * z - r2) * y, 5 * z ** 3 - 3 * z * r2,
                         (5 * z * z - r2) * x, x * x * z - y * y * z, x ** 3 - 3 * x * y * y,
                         dw / (2 * np.pi * GAMMA) if dw_prec else torch.zeros_like(x)], dim=1)
    h = np.asarray(seq.h, dtype=np.float64).copy()
    if not ho0:
        h[0] = 0
    if not ho1:
        h[1], h[2], h[3] = seq.gx, seq.gy, seq.gz
    if not ho2:
        h[4:9] = 0
    if not ho3:
        h[9:16] = 0
    coef = T(np.vstack([h, np.ones((1, h.shape[1]))]))
    dt = T(seq.dt)
    gx, gy, gz, df, psi = T(seq.gx), T(seq.gy), T(seq.gz), T(seq.df), T(seq.psi)
    b1 = T(np.asarray(seq.b1), ct)
    adc = np.asarray(seq.adc, dtype=bool)
    nadc = sum(int(adc[f + 1:l + 1].sum()) for f, l in w.parts)
    sig = torch.zeros((nadc, csm.shape[1]), dtype=ct, device=dev)
    mxy0 = torch.zeros_like(x, dtype=ct)
    mz0 = rho.clone()
    c_neg = -2 * np.pi * GAMMA
    eps = float(np.finfo(np.float64 if dtype == "f64" else np.float32).eps)
    # block plan (ADC columns as slices, or index tensors built before the timed region)
    blocks = {}
    for (f, l), exc in zip(w.parts, w.excitation):
        if exc:
            continue
        a = f
        while a < l:
            b = min(l, a + block)
            cols = np.flatnonzero(adc[a + 1:b + 1])
            if cols.size and np.array_equal(cols, np.arange(cols[0], cols[0] + cols.size)):
                sel = slice(int(cols[0]), int(cols[0]) + cols.size)
            else:
                sel = torch.as_tensor(cols, device=dev) if cols.size else None
            blocks[a] = (b, sel, int(cols.size))
            a = b
    def body():
        _run(mxy0, mz0)

    def _run(mxy, mz):
        row = 0
        for (f, l), exc in zip(w.parts, w.excitation):
            if exc:
                mxy = mxy * torch.polar(torch.ones_like(x), -psi[f].expand_as(x))
                off = dw / (2 * np.pi * GAMMA) if dw_exc else torch.zeros_like(x)
                for n in range(f, l):
                    bz = (gx[n] * x + gy[n] * y) + gz[n] * z + (off - df[n] / GAMMA)
                    bb = torch.sqrt(b1[n].abs() ** 2 + bz * bz)
                    bb = torch.where(bb == 0, torch.full_like(bb, eps), bb)
                    half = c_neg * (bb * dt[n]) / 2
                    sh, ch = torch.sin(half), torch.cos(half)
                    al = torch.complex(ch, -(bz / bb) * sh)
                    be = torch.complex((b1[n].imag / bb) * sh, -(b1[n].real / bb) * sh)
                    nxy = 2 * al.conj() * be * mz + al.conj() ** 2 * mxy - be ** 2 * mxy.conj()
                    nmz = (al.abs() ** 2 - be.abs() ** 2) * mz - 2 * (al * be * mxy.conj()).real
                    e1 = torch.exp(-dt[n] / T1)
                    mxy = nxy * torch.exp(-dt[n] / T2)
                    mz = nmz * e1 + rho * (1 - e1)
                    if adc[n + 1]:
                        s_ = mxy * torch.polar(torch.ones_like(x), psi[n + 1].expand_as(x))
                        sig[row] = s_ @ csm
                        row += 1
                mxy = mxy * torch.polar(torch.ones_like(x), psi[l].expand_as(x))
                continue
            a = f
            while a < l:
                b, sel, ncol = blocks[a]
                bz = basis @ coef[:, a:b + 1]
                d = dt[a:b]
                phi = torch.cumsum((bz[:, :-1] + bz[:, 1:]) * (-np.pi * GAMMA * d), dim=1)
                tr = torch.cumsum(d, dim=0)
                mblk = mxy[:, None] * torch.exp(torch.complex(-tr[None, :] / T2[:, None], phi))
                if ncol:
                    states = mblk[:, sel]
                    sig[row:row + ncol] = states.transpose(0, 1) @ csm
                    row += ncol
                mxy = mblk[:, -1]
                e1 = torch.exp(-tr[-1] / T1)
                mz = mz * e1 + rho * (1 - e1)
                a = b
    ms = None
    if graph:
        torch.cuda.synchronize()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            e0, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(side)
            body()  # the eager run, also the warm-up before the capture (cuBLAS handles, workspaces)
            e1_.record(side)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        if times is not None:
            times["eager_ms"] = e0.elapsed_time(e1_)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            body()
        torch.cuda.synchronize()
        sig.zero_()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        g.replay()
        stop.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(stop)
        if times is not None:
            times["graph_ms"] = ms
        del g
    elif time_it:
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        body()
        stop.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(stop)
    else:
        body()
    return sig.cpu().numpy(), ms


def reference_gpu_leg(w, fused_sig, fused_ms: float, units: float) -> dict:
    """Time ``reference_gpu_equivalent`` once per precision on the full
    workload (after a warm-up on a spin subsample) and compare its FP64 signal
    with the fused kernel's."""
    import torch
    out = {"design": "the reference's GPU path restated with torch/cuBLAS: per block of <= 32 nodes a basis x "
                     "coefficient GEMM for the field, trapezoid phase, materialised ADC states, and a complex "
                     "cuBLAS GEMM states^T csm (kernels/HighOrderGPU.jl:6-178); host loop over blocks",
           "block_nodes": 32}
    try:
        small = _workload(50)
        for dt in ("f32", "f64"):
            reference_gpu_equivalent(small, dt)
            tm = {}
            sig, ms = reference_gpu_equivalent(w, dt, graph=True, times=tm)
            out[dt] = {"ms": ms, "units_per_s": units / (ms / 1e3), "fused_speedup": ms / fused_ms,
                       "host_loop_ms": tm.get("eager_ms"), "timing": "CUDA-graph replay of the whole block loop"}
            if dt == "f64":
                fused = fused_sig.transpose(0, 1).cpu().numpy()
                out[dt]["nrmse_fused_vs_this"] = float(np.linalg.norm(fused - sig) / np.linalg.norm(sig))
            del sig
            torch.cuda.empty_cache()
    except Exception as e:  # the comparator must not take the bench line down
        out["error"] = f"{type(e).__name__}: {e}"
    return out


def _pinned(torch, a: np.ndarray) -> np.ndarray:
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    out = t.numpy().view(a.dtype).reshape(a.shape, order="F" if a.flags.f_contiguous and not a.flags.c_contiguous
                                          else "C")
    out[...] = a  # the view's .base chain keeps the pinned tensor alive
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="homs", choices=["homs", "reference"])
    ap.add_argument("--mode", default="split", choices=["split", "plain"])
    ap.add_argument("--config", type=int, default=CONFIG_INDEX, choices=[0, 1, 2, 3],
                    help="benchmark configuration (2: the 3D 32-coil workload, the default bench line)")
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"],
                    help="dtype of the arrays (split mode computes in FP64 either way)")
    ap.add_argument("--spin-stride", type=int, default=1,
                    help="run every k-th spin of the workload (small cases for profiling; bench lines use 1)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparator on the same workload")
    ap.add_argument("--no-configs", action="store_true", help="skip the other workloads (2D 1-coil, 2D 8-coil, TR loop)")
    ap.add_argument("--no-kspace", action="store_true", help="skip the encoding-export measurement")
    ap.add_argument("--no-refgpu", action="store_true",
                    help="skip timing the restatement of the reference's GPU design (reference_gpu_equivalent)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_homs(args)


if __name__ == "__main__":
    sys.exit(main())
