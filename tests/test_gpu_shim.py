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


def test_cpp_driver_output_files(lib_built, tmp_path):
    """The driver's output path through the shim's FalmIO and TAvg (every step,
    averaging from step 3): the u + p vector files, the averaged files, the
    index file and the control-volume file. The last snapshot holds the final
    fields; the last averaged file is the mean of the snapshots of steps 3..6."""
    import json
    from falm_b200 import api
    case = cases.small_channel(32, 20, 20, intensity=0.0)
    steps = 6
    cpath, opath = str(tmp_path / "case.bin"), str(tmp_path / "out.bin")
    write_case(cpath, case, steps, 6, 0.0)
    prefix = str(tmp_path / "run")
    r = subprocess.run([DRIVER, cpath, opath, prefix, "1", "3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    n, g = case.grid.n, case.grid
    raw = np.fromfile(opath, dtype="<f8")
    u_end, p_end = raw[:3 * n], raw[6 * n:7 * n]
    names = sorted(os.listdir(tmp_path))
    assert [x for x in names if x.startswith("run_0")] == [f"run_000000_{it:010d}" for it in range(1, 7)]
    assert [x for x in names if x.startswith("run_tavg")] == [f"run_tavg_000000_{it:010d}" for it in range(3, 7)]
    snaps = {}
    for it in range(1, 7):
        hd, data = api.read_vector_file(tmp_path / f"run_000000_{it:010d}")
        assert (hd["ncol"], hd["step"], hd["dsize"], hd["time"]) == (4, it, 8, it * case.dt)
        snaps[it] = data
    np.testing.assert_array_equal(snaps[6][:3].ravel(), u_end)
    np.testing.assert_array_equal(snaps[6][3].ravel(), p_end)
    _, avg6 = api.read_vector_file(tmp_path / "run_tavg_000000_0000000006")
    mean = np.mean([snaps[it] for it in range(3, 7)], axis=0)
    assert rel_l2(avg6[:3].ravel(), mean[:3].ravel()) < 1e-13
    assert rel_l2(avg6[3].ravel(), mean[3].ravel()) < 1e-13
    idx = json.loads((tmp_path / "run.json").read_text())
    assert [(s["step"], s.get("timeAvg", 0)) for s in idx["outputSteps"]] == [(1, 0), (2, 0), (3, 1), (4, 1), (5, 1), (6, 1)]
    assert idx["global"] == list(g.interior) and idx["guidePoint"] == g.gc
    assert api.read_cv_file(tmp_path / "run.cv")[0] == (g.sx, g.sy, g.sz, g.gc)
