"""Regenerate the golden fixtures in this directory.

Inputs are the reference's closed-form fixtures (test/support/high_order_workload.jl,
test/support/compatibility_workload.jl) rebuilt by homs.workloads; outputs are
the FP64 CPU oracle's (oracle/homs_oracle.c, one thread, so the summation
order is fixed).  Known-answer values of the reference's tests are stored
beside them.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "highordermrisim.jl_b200"))
sys.path.insert(0, ROOT)

from homs import workloads as W  # noqa: E402
from homs.model import GAMMA, BlochHighOrder  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cases():
    out = {}
    for nc in (1, 3, 32):
        obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=nc)
        out[f"hw259_c{nc}_prec"] = (obj, seq, [(0, 32)], [False], "1111", st)
        obj, seq, st = W.high_order_workload(nspins=259, nsteps=32, ncoils=nc, rf=True)
        out[f"hw259_c{nc}_rf"] = (obj, seq, [(0, 32)], [True], "1111", st)
    obj = W.compatibility_phantom()
    seq, parts, exc, _ = W.compatibility_sequence()
    out["compat_0000"] = (obj, seq, parts, exc, "0000", None)
    seq, parts, exc, _ = W.compatibility_sequence(h0_readout=20 / GAMMA)
    out["compat_1000_h0"] = (obj, seq, parts, exc, "1000", None)
    obj, seq, parts, exc = W.rf_acquisition_workload(3, 2, 11)
    out["rfacq_3_2_11"] = (obj, seq, parts, exc, "1111", None)
    return out


def main():
    O.build()
    arrays = {}
    for name, (obj, seq, parts, exc, mask, st) in cases().items():
        flags = BlochHighOrder(mask).flags
        mxy0 = None if st is None else st.xy
        mz0 = None if st is None else st.z
        sig, xy, z = O.simulate_c(obj, seq, parts, exc, flags, mxy0, mz0, nthreads=1)
        arrays[f"{name}/sig"] = sig
        arrays[f"{name}/xy"] = xy
        arrays[f"{name}/z"] = z
    np.savez_compressed(os.path.join(HERE, "oracle_fixtures.npz"), **arrays)
    print(f"wrote {len(arrays)} arrays")


if __name__ == "__main__":
    main()
