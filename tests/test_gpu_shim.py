"""The C++ class shim (include/falm_b200.hpp) as a drop-in for the reference's
solver classes: falm_b200/nedo_driver runs the time loop of app/nedo/main.cpp
through FalmCFD / FalmEq / FalmMV / Alm::AlmHandler method calls, and its
fields after 6 steps match the CPU oracle (FP64, fixed-iteration mode so the
stopping rule plays no part: relative L2 <= 1e-10)."""
import os
import struct
import subprocess

import numpy as np
import pytest

from falm_b200 import cases
from tests.helpers import faces, interior, rel_l2
from tests.test_gpu_step import run_oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "falm_b200", "nedo_driver")


def write_case(path, case, steps, maxit, tol):
    g = case.grid
    adv = {"Upwind1": 0, "Upwind3": 1, "QUICK": 2, "UTOPIA": 3, "KK": 4}[case.adv]
    sgs = {"Empty": 0, "Smagorinsky": 1, "CSM": 2}[case.sgs]
    pc = {"Jacobi": 1, "SOR": 2}[case.pc]
    st = cases.initial_state(case)
    with open(path, "wb") as f:
        f.write(struct.pack("<12i", g.sx, g.sy, g.sz, g.gc, steps, maxit, case.pc_maxit, adv, sgs, case.bc, pc,
                            1 if case.alm is not None else 0))
        f.write(struct.pack("<6d", case.Re, case.Cs, case.dt, tol, case.pc_relax, case.u_inlet))
        for a in (g.x, g.y, g.z, g.hx, g.hy, g.hz, st["u"]):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        if case.alm is not None:
            a = case.alm
            f.write(struct.pack("<4i", a.n_blade, a.n_ap_per_blade, a.n_attack, int(a.angle_type[0])))
            f.write(struct.pack("<3d", a.radius, a.hub_radius, a.euler_eps))
            k = a.arrays()
            for arr in (k["base"][:3], k["hub"][:3], k["tip_rate"][:1], k["motion"][:3], k["ap_r"], k["ap_chord"],
                        k["ap_twist"], k["attack"], k["cl"], k["cd"]):
                f.write(np.ascontiguousarray(arr, dtype="<f8").tobytes())


@pytest.mark.parametrize("name", ["channel", "cavity"])
def test_cpp_driver_matches_oracle(oracle, lib_built, tmp_path, name):
    if name == "channel":
        case = cases.small_channel(32, 20, 20, intensity=0.0)
    else:
        case = cases.cavity(16)
    steps, maxit, tol = 6, 6, 0.0
    cpath, opath = str(tmp_path / "case.bin"), str(tmp_path / "out.bin")
    write_case(cpath, case, steps, maxit, tol)
    r = subprocess.run([DRIVER, cpath, opath], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert len(r.stdout.strip().splitlines()) == steps
    n = case.grid.n
    raw = np.fromfile(opath, dtype="<f8")
    got = {"u": raw[:3 * n], "uu": raw[3 * n:6 * n], "p": raw[6 * n:7 * n], "nut": raw[7 * n:8 * n]}
    stats = raw[8 * n:].reshape(steps, 5)
    ref, rs = run_oracle(oracle, case, steps, maxit=maxit, tol=tol)
    g = case.grid
    assert rel_l2(interior(got["u"], g, 3), interior(ref["u"], g, 3)) < 1e-10
    assert rel_l2(faces(got["uu"], g), faces(ref["uu"], g)) < 1e-10
    assert rel_l2(interior(got["p"], g), interior(ref["p"], g)) < 1e-10
    assert rel_l2(interior(got["nut"], g), interior(ref["nut"], g)) < 1e-10
    for q in range(steps):
        assert stats[q, 0] == rs[q]["it"]
        if case.alm is not None:
            assert stats[q, 3] == pytest.approx(rs[q]["torque"][0], rel=1e-10)
