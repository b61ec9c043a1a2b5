"""The reference's demo3D and demo2D workloads on one GPU.

demo3D/1_load_seq.jl builds the sequence (a Pulseq 1.4 3D stack of spirals,
40 TRs of 500 ms, 35 partitions x 3,800 ADC samples, with field-camera
gradients in the readouts), demo3D/2_load_phantom.jl the phantom (the
0.5 mm brain class volume resampled to the sequence's 100 x 100 x 35 grid
at 2 mm around z = 20 mm, the real 32-channel receive map and the real
off-resonance map, 1.5 T tissue), and demo3D/3_run_sim.jl runs
BlochHighOrder("1111") with FP32 arrays.  Two steps:

    python bench_demo.py stage --demo-dir DEMO3D --phantom-dir PHANTOM --out DIR
        (CPU) copies the three demo files and writes the phantom's class and
        off-resonance volumes, resampled to the target grid, and the source
        receive map to DIR (about 40 MB).
    python bench_demo.py run --staged DIR [--runs 4] [--modes split_f32,...]
        (GPU) builds the sequence and the phantom, prepares one plan per
        mode (split and plain, FP32 and FP64 arrays), times repeated plan
        runs (host wall time of ``Plan.run``, signal copied to host memory
        included; the best of ``--runs``) and prints one JSON line with the
        times, spin*sample*coil/s and each mode's NRMSE against plain FP64.

DEMO3D holds Spiral_2p0x2p0x2p0_100x100x35_1x4_int1_9p5ms_tr500_te5p0{.seq,
.mat,_skope.mat}; PHANTOM holds brain3D_0.5_0.5_0.5.mat, csm/csm_4p0.mat and
b0map/b0_4p0.mat, as in the reference's source tree.  ``--workload demo2d``
(both steps, with the demo2D directory) runs demo2D/1_load_inputs.jl and
Sim2D.jl instead: 7T_1p0_200_r4{.seq,.mat}, a 200 x 200 x 1 slice at
1 x 1 x 4 mm, B0 and T2 switched off as the demo does.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if os.path.join(ROOT, "highordermrisim.jl_b200") not in sys.path:
    sys.path.insert(0, os.path.join(ROOT, "highordermrisim.jl_b200"))

NAME = "Spiral_2p0x2p0x2p0_100x100x35_1x4_int1_9p5ms_tr500_te5p0"
NAME_2D = "7T_1p0_200_r4"
# target grid (resolution, matrix, location), files, and the demo's B0 / T2 switches
WORKLOADS = {
    "demo3d": dict(res=(0.002, 0.002, 0.002), matrix=(100, 100, 35), location=(0.0, 0.0, 0.02),
                   files=(NAME + ".seq", NAME + ".mat", NAME + "_skope.mat"), b0=True, t2=True),
    "demo2d": dict(res=(0.001, 0.001, 0.004), matrix=(200, 200, 1), location=(0.0, 0.0, 0.0),
                   files=(NAME_2D + ".seq", NAME_2D + ".mat"), b0=False, t2=False),
}
TARGET_RES, TARGET_MATRIX, LOCATION = (WORKLOADS["demo3d"][k] for k in ("res", "matrix", "location"))


def stage(demo_dir: str, phantom_dir: str, out: str, workload: str = "demo3d") -> None:
    import scipy.io as sio

    from homs.phantom import resample_b0, resample_labels
    w = WORKLOADS[workload]
    os.makedirs(out, exist_ok=True)
    for f in w["files"]:
        shutil.copyfile(os.path.join(demo_dir, f), os.path.join(out, f))
    brain = sio.loadmat(os.path.join(phantom_dir, "brain3D_0.5_0.5_0.5.mat"))["data"]
    labels = resample_labels(brain, (0.5e-3,) * 3, w["res"], w["matrix"], w["location"])
    b0 = sio.loadmat(os.path.join(phantom_dir, "b0map", "b0_4p0.mat"))["b0"]
    fieldmap = resample_b0(b0, (4e-3,) * 3, w["res"], w["matrix"], w["location"])
    csm = sio.loadmat(os.path.join(phantom_dir, "csm", "csm_4p0.mat"))["csm"].astype(np.complex64)
    np.savez(os.path.join(out, workload + "_phantom_volumes.npz"), labels=labels,
             fieldmap=fieldmap.astype(np.float32), csm_source=csm)


def _nrmse(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


MODES = {"split_f32": ("f32", "split"), "split_f64": ("f64", "split"), "plain_f64": ("f64", "plain"),
         "plain_f32": ("f32", "plain")}


def run(staged: str, runs: int = 4, modes=tuple(MODES), workload: str = "demo3d") -> dict:
    from homs import Context, prepare_simulation
    from homs.demo_inputs import demo2d_sequence, demo3d_sequence
    from homs.model import BlochHighOrder
    from homs.phantom import brain_phantom, resample_csm
    from homs.sequence import discretize, get_adc_phase_compensation

    w = WORKLOADS[workload]
    out = {"workload": {"demo3d": "demo3D: Pulseq 3D stack of spirals with field-camera gradients, brain phantom "
                                  "with real 32-channel receive and off-resonance maps",
                        "demo2d": "demo2D: Pulseq 2D 7T spiral with the stitched field measurement, brain slice "
                                  "with the real 32-channel receive map, B0 and T2 off"}[workload]}
    t0 = time.perf_counter()
    paths = [os.path.join(staged, f) for f in w["files"]]
    hoseq = demo3d_sequence(*paths) if workload == "demo3d" else demo2d_sequence(*paths)
    out["sequence_build_s"] = time.perf_counter() - t0
    vol = np.load(os.path.join(staged, workload + "_phantom_volumes.npz"))
    csm = resample_csm(vol["csm_source"], (4e-3,) * 3, w["res"], w["matrix"], w["location"])
    ctx = Context(0)
    t0 = time.perf_counter()
    obj = brain_phantom(vol["labels"], w["res"], fieldstrength="1.5T",
                        fieldmap=vol["fieldmap"].astype(np.float64), csm=csm, context=ctx)
    out["phantom_build_s"] = time.perf_counter() - t0
    if not w["b0"]:
        obj.dw[:] = 0.0
    if not w["t2"]:
        obj.T2[:] = np.inf
    t0 = time.perf_counter()
    seqd = discretize(hoseq)
    out["discretize_s"] = time.perf_counter() - t0
    out.update(spins=len(obj), coils=obj.ncoils, nodes=seqd.nnodes, adc=int(seqd.adc.sum()),
               rf_intervals=int(seqd.excitation.sum()))
    out["units"] = out["spins"] * out["adc"] * out["coils"]
    method = BlochHighOrder("1111", True, True)
    sig = {}
    for name in modes:
        prec, mode = MODES[name]
        src = obj if prec == "f64" else obj.astype(np.float32)
        params = {"sim_method": method, "precision": prec, "homs_precision": mode}
        with prepare_simulation(src, hoseq, sim_params=params, context=ctx) as plan:
            s = plan.run()
            best = float("inf")
            for _ in range(runs):
                t0 = time.perf_counter()
                s = plan.run()
                best = min(best, time.perf_counter() - t0)
        sig[name] = s[:, :, 0].astype(np.complex128)
        out[name + "_ms"] = best * 1e3
        out[name + "_units_per_s"] = out["units"] / best
    for name in sig:
        if name != "plain_f64" and "plain_f64" in sig:
            out[name + "_nrmse_vs_plain_f64"] = _nrmse(sig[name], sig["plain_f64"])
    if "split_f32" in sig and "plain_f64" in sig:
        # the FP32-array run against plain FP64 on the same FP32-rounded inputs: the split path's own error
        seqd32 = seqd.astype(np.float32).astype(np.float64)
        obj32 = obj.astype(np.float32).astype(np.float64)
        params = {"sim_method": method, "precision": "f64", "homs_precision": "plain"}
        with prepare_simulation(obj32, seqd32, sim_params=params, context=ctx) as plan:
            ref32 = plan.run()[:, :, 0] * get_adc_phase_compensation(hoseq).astype(np.complex128)[:, None]
        out["split_f32_nrmse_vs_plain_f64_same_inputs"] = _nrmse(sig["split_f32"], ref32)
    ctx.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("stage")
    s.add_argument("--workload", choices=tuple(WORKLOADS), default="demo3d")
    s.add_argument("--demo-dir", required=True)
    s.add_argument("--phantom-dir", required=True)
    s.add_argument("--out", required=True)
    r = sub.add_parser("run")
    r.add_argument("--workload", choices=tuple(WORKLOADS), default="demo3d")
    r.add_argument("--staged", required=True)
    r.add_argument("--runs", type=int, default=4)
    r.add_argument("--modes", default=",".join(MODES), help="comma-separated subset of " + ", ".join(MODES))
    a = ap.parse_args(argv)
    if a.cmd == "stage":
        stage(a.demo_dir, a.phantom_dir, a.out, a.workload)
    else:
        modes = tuple(m for m in a.modes.split(",") if m)
        if not modes or any(m not in MODES for m in modes):
            ap.error("--modes takes a comma-separated subset of " + ", ".join(MODES))
        print(json.dumps(run(a.staged, a.runs, modes, a.workload)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
