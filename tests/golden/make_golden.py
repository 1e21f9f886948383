"""Generate golden vectors from the reference's OWN CUDA step.

Runs oracle/_ref/libfalmref.so (the reference's sources compiled by
oracle/Makefile) on small seeded cases and stores the fields after 3 steps
(fixed-iteration mode: maxit 4, tol 0) as tests/golden/<case>.npz.  Needs a GPU
and the prebuilt oracle/_ref; run from the repository root:

    python tests/golden/make_golden.py [outdir]

The CPU test tests/test_golden.py checks the oracle against these files.
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from falm_b200 import cases  # noqa: E402
from oracle.oracle import CaseStruct, RefStep  # noqa: E402

STEPS, MAXIT, TOL = 3, 4, 0.0


def golden_cases():
    ch = cases.small_channel(16, 12, 12, cells_per_radius=3, intensity=0.0, n_ap_per_blade=5)
    cav = cases.cavity(8)
    return {"channel": ch, "cavity": cav}


def pack(case, fields, stats):
    g = case.grid
    gc = g.gc

    def view(a, nc):
        return a.reshape(nc, g.sz, g.sy, g.sx)
    return {
        "u": view(fields["u"], 3)[:, gc:-gc, gc:-gc, gc:-gc].copy(),
        "uu": view(fields["uu"], 3)[:, gc - 1:-gc, gc - 1:-gc, gc - 1:-gc].copy(),
        "p": view(fields["p"], 1)[:, gc:-gc, gc:-gc, gc:-gc].copy(),
        "nut": view(fields["nut"], 1)[:, gc:-gc, gc:-gc, gc:-gc].copy(),
        "it": np.array([s["it"] for s in stats]),
        "torque": np.array([s["torque"][0] if s["torque"] else 0.0 for s in stats]),
        "thrust": np.array([s["thrust"][0] if s["thrust"] else 0.0 for s in stats]),
        "divnorm": np.array([s["divnorm"] for s in stats]),
    }


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name, case in golden_cases().items():
        cs = CaseStruct(case, use_inflow=False, maxit=MAXIT, tol=TOL)
        ref = RefStep(cs, tempfile.mkdtemp(prefix="falmgold_"))
        st = cases.initial_state(case)
        ref.set("U", st["u"])
        ref.op("UTOUU")
        ref.op("SGS")
        stats = [ref.step((q + 1) * case.dt) for q in range(STEPS)]
        fields = {k: ref.get(n) for k, n in (("u", "U"), ("uu", "UU"), ("p", "P"), ("nut", "NUT"))}
        ref.close()
        np.savez_compressed(os.path.join(outdir, f"{name}.npz"), **pack(case, fields, stats))
        print(name, "written", stats[-1])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"))
