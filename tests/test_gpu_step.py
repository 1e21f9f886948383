"""Whole-step parity: falm_step (CUDA, through the C ABI) against the CPU oracle's
restatement of app/nedo/main.cpp:150-204 and app/lid3d/main.cpp:121-168.

FP64: relative L2 <= 1e-10 on u, uu, p, nut after 10 steps (in fixed-iteration
mode, and in convergence mode with BiCGStab iteration counts within +-1).
Mixed (FP32 storage, FP64 reductions): relative L2 of u <= 2e-4 and of p <= 5e-3
after 10 steps, rotor power and thrust within 0.5%, div norm within the tolerance."""
import numpy as np
import pytest

from falm_b200 import cases
from tests.helpers import dev, faces, host, interior, make_ctx, rel_l2

pytestmark = pytest.mark.gpu


def run_oracle(oracle, case, steps, maxit=None, tol=None):
    from oracle.oracle import CaseStruct
    cs = CaseStruct(case, maxit=maxit, tol=tol)
    m = oracle.setup(cs)
    st = cases.initial_state(case)
    oracle.init_state(cs, m, st)
    stats = [oracle.step(cs, st, m, (it + 1) * case.dt) for it in range(steps)]
    return st, stats


def run_gpu(case, steps, precision="fp64", fuse_alm=True, maxit=None, tol=None):
    ctx = make_ctx(case, precision)
    if maxit is not None or tol is not None:
        ctx.eq_init(maxit or case.maxit, case.tol if tol is None else tol, case.pc, case.pc_maxit, case.pc_relax)
    st0 = cases.initial_state(case)
    u, uu, p, nut = dev(ctx, st0["u"]), ctx.field(3), ctx.field(1), ctx.field(1)
    ctx.utouu(u, uu)
    ctx.sgs(u, nut)
    ff = None if (fuse_alm and case.alm is not None) else ctx.field(3)
    stats = [ctx.step(u, uu, p, nut, ff, case.dt, (it + 1) * case.dt) for it in range(steps)]
    return {"u": host(u), "uu": host(uu), "p": host(p), "nut": host(nut)}, stats, ctx


def compare(case, a, b):
    g = case.grid
    return {
        "u": rel_l2(interior(a["u"], g, 3), interior(b["u"], g, 3)),
        "uu": rel_l2(faces(a["uu"], g), faces(b["uu"], g)),
        "p": rel_l2(interior(a["p"], g), interior(b["p"], g)),
        "nut": rel_l2(interior(a["nut"], g), interior(b["nut"], g)),
    }


def small_cases():
    ch = cases.small_channel(32, 20, 20, intensity=0.05).with_inflow(nb=8)
    cav = cases.cavity(16)
    cav.tol = 1e-10
    # wide enough (nx >= 64) for every plane stream, including the 7-point one
    wide = cases.small_channel(72, 20, 16, intensity=0.05).with_inflow(nb=8)
    # an odd interior width: rows whose pitch is not a multiple of 16 bytes,
    # so every plane stream gives way to the row kernels
    odd = cases.small_channel(33, 19, 15, intensity=0.05).with_inflow(nb=8)
    return {"channel": ch, "cavity": cav, "wide": wide, "odd": odd}


@pytest.mark.parametrize("name", ["channel", "cavity", "wide", "odd"])
def test_step_fp64_fixed_iterations(oracle, lib_built, name):
    case = small_cases()[name]
    ref, rs = run_oracle(oracle, case, 10, maxit=6, tol=0.0)
    got, gs, _ = run_gpu(case, 10, maxit=6, tol=0.0)
    err = compare(case, got, ref)
    for k, v in err.items():
        assert v < 1e-10, (k, v, err)
    for a, b in zip(gs, rs):
        assert a["it"] == b["it"]
        assert a["divnorm"] == pytest.approx(b["divnorm"], rel=1e-6, abs=1e-18)
        for x, y in zip(a["torque"] + a["thrust"], b["torque"] + b["thrust"]):
            assert x == pytest.approx(y, rel=1e-10)


def oracle_spread(oracle, case, steps, eps=1e-15, seed=1):
    """How far the oracle's own fields move when its initial velocity is scaled
    by (1 + eps * N(0, 1)) cell by cell: the rounding sensitivity of the
    fixed-iteration step map for this case."""
    from oracle.oracle import CaseStruct
    cs = CaseStruct(case, maxit=6, tol=0.0)
    m = oracle.setup(cs)
    st = cases.initial_state(case)
    st["u"] = st["u"] * (1 + eps * np.random.default_rng(seed).standard_normal(st["u"].shape))
    oracle.init_state(cs, m, st)
    for it in range(steps):
        oracle.step(cs, st, m, (it + 1) * case.dt)
    return st


@pytest.mark.parametrize("pc_maxit", [2, 3, 4])
def test_step_fp64_fixed_iterations_jacobi(oracle, lib_built, pc_maxit):
    """Jacobi preconditioning through the step: the face-velocity kernel's fused
    first residual writes the first sweep into the buffer from which the sweeps
    ping-pong to pp (xp for an even sweep count, pp for an odd one).

    With 3 sweeps this case's BiCGStab runs close to a breakdown: a 1e-15
    relative perturbation of the oracle's own input moves its pressure by about
    6e-8 (against 2e-15 at 2 or 4 sweeps). There the bound is that measured
    spread of the oracle itself, otherwise 1e-10."""
    case = small_cases()["wide"]
    case.pc, case.pc_maxit = "Jacobi", pc_maxit
    ref, rs = run_oracle(oracle, case, 5, maxit=6, tol=0.0)
    got, gs, _ = run_gpu(case, 5, maxit=6, tol=0.0)
    err = compare(case, got, ref)
    spread = compare(case, oracle_spread(oracle, case, 5), ref)
    for k, v in err.items():
        assert v < max(1e-10, spread[k]), (k, v, err, spread)
    for a, b in zip(gs, rs):
        assert a["it"] == b["it"]


@pytest.mark.parametrize("name", ["channel", "cavity"])
def test_step_fp64_converged(oracle, lib_built, name):
    case = small_cases()[name]
    ref, rs = run_oracle(oracle, case, 10)
    got, gs, _ = run_gpu(case, 10)
    for a, b in zip(gs, rs):
        assert abs(a["it"] - b["it"]) <= 1
        assert a["err"] <= case.tol or a["it"] == case.maxit
    err = compare(case, got, ref)
    for k, v in err.items():
        assert v < 1e-9, (k, v, err)


def test_step_alm_fused_equals_stored_force(lib_built):
    """The in-kernel ALM projection and the stored ff field give the same step."""
    case = small_cases()["channel"]
    a, sa, _ = run_gpu(case, 3, fuse_alm=True)
    b, sb, _ = run_gpu(case, 3, fuse_alm=False)
    for k in a:
        assert rel_l2(a[k], b[k]) < 1e-13, k


def test_step_mixed_vs_fp64_oracle(oracle, lib_built):
    case = small_cases()["channel"]
    case.tol = 1e-8
    ref, rs = run_oracle(oracle, case, 10)
    got, gs, _ = run_gpu(case, 10, precision="mixed")
    err = compare(case, got, ref)
    assert err["u"] < 2e-4, err
    assert err["uu"] < 2e-4, err
    # the pressure is determined to the solver tolerance only (both runs stop at
    # ||r||/N <= tol with different iterates); velocities are the physical check
    assert err["p"] < 2e-2, err
    for a, b in zip(gs, rs):
        assert a["err"] <= case.tol * 1.0000001 or a["it"] >= case.maxit
        assert a["torque"][0] == pytest.approx(b["torque"][0], rel=5e-3)
        assert a["thrust"][0] == pytest.approx(b["thrust"][0], rel=5e-3)
        assert a["divnorm"] <= max(10 * b["divnorm"], 1e-9)


def test_step_cavity_mixed(oracle, lib_built):
    case = small_cases()["cavity"]
    case.tol = 1e-8
    ref, rs = run_oracle(oracle, case, 10)
    got, gs, _ = run_gpu(case, 10, precision="mixed")
    err = compare(case, got, ref)
    assert err["u"] < 2e-4, err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_streamed_inlet_planes_match_inflow_box(lib_built, precision):
    """falm_bc_set_inlet_plane: run b takes, as a pinned host plane copied before
    each step, the inlet plane that run a's step sampled from the inflow box on
    the device (read back from a's inlet ghost layer), and makes the same steps
    bit for bit. A plane set twice before a step is replaced by the second call;
    a step without a plane samples the box again."""
    import torch
    from falm_b200.driver import Simulation
    case = small_cases()["channel"]
    g = case.grid
    sx, sy, sz, gc = g.sx, g.sy, g.sz, g.gc
    a, b = Simulation(case, precision), Simulation(case, precision)

    def inlet(sim):
        u = host(sim.u).reshape(3, sz, sy, sx)
        return np.ascontiguousarray(u[:, gc:sz - gc, gc:sy - gc, gc - 1])

    keep = []
    for q in range(5):
        sa = a.step()
        plane = torch.from_numpy(inlet(a)).pin_memory()
        keep.append(plane)
        if q == 2:
            wrong = torch.zeros_like(plane).pin_memory()
            keep.append(wrong)
            b.ctx.set_inlet_plane(wrong)
        b.ctx.set_inlet_plane(plane)
        sb = b.step()
        assert sa["it"] == sb["it"]
        for x, y in ((a.u, b.u), (a.p, b.p), (a.uu, b.uu), (a.nut, b.nut)):
            assert np.array_equal(host(x), host(y)), q
    a.step(), b.step()
    assert np.array_equal(host(a.u), host(b.u))


def test_step_launch_count_and_statuses(lib_built):
    case = small_cases()["channel"]
    got, gs, ctx = run_gpu(case, 2)
    assert ctx.launches() > 0
    for s in gs:
        assert s["status"] == 0 and s["outer"] == 1
        assert np.isfinite(s["divnorm"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["channel", "cavity", "wide"])
def test_device_loop_equals_host_loop(lib_built, monkeypatch, precision, name):
    """The step recorded as one CUDA graph, its solver loops conditional while
    nodes (the default; FALM_B200_GRAPH=1), runs the same kernels in the same
    order as the host-driven step, whose loop queues iterations in batches
    between reads of the convergence flag (FALM_B200_GRAPH=0): the
    same iteration counts and bitwise the same fields, in convergence mode
    (where the loop's exit matters) and in fixed-iteration mode; "wide" (72
    cells across) runs every TMA plane stream, recorded with its tensor maps."""
    case = small_cases()[name]
    for maxit, tol in ((None, None), (6, 0.0)):
        outs = []
        for mode in ("0", "1"):
            monkeypatch.setenv("FALM_B200_GRAPH", mode)
            got, st, ctx = run_gpu(case, 4, precision=precision, maxit=maxit, tol=tol)
            ctx.close()
            outs.append((got, [x["it"] for x in st], [x["outer"] for x in st]))
        assert outs[0][1] == outs[1][1] and outs[0][2] == outs[1][2], (outs[0][1:], outs[1][1:])
        for k in outs[0][0]:
            assert np.array_equal(outs[0][0][k], outs[1][0][k]), k


@pytest.mark.parametrize("shape", [(40, 20, 72), (72, 20, 40)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_tma_matches_row_kernels_multichunk(lib_built, monkeypatch, precision, shape):
    """Several z chunks per column and partial x/y tiles: the TMA plane streams
    and the row kernels give the same steps (the 7-point stream's 64-wide tile
    needs nx >= 64)."""
    case = cases.small_channel(*shape, intensity=0.05).with_inflow(nb=8)
    outs = []
    for no_tma in ("1", "0"):
        monkeypatch.setenv("FALM_B200_NO_TMA", no_tma)
        got, st, _ = run_gpu(case, 3, precision=precision, maxit=4, tol=0.0)
        outs.append(got)
    # FP32: the two kernel families round differently; the solver carries that
    # into the pressure (determined to the iteration's accuracy only)
    tol = {"u": 1e-12, "uu": 1e-12, "p": 1e-12, "nut": 1e-12} if precision == "fp64" else \
        {"u": 1e-5, "uu": 1e-5, "p": 1e-3, "nut": 1e-5}
    for k in outs[0]:
        assert rel_l2(outs[1][k], outs[0][k]) < tol[k], (k, rel_l2(outs[1][k], outs[0][k]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_snapshots_and_time_average(lib_built, tmp_path, precision):
    """Snapshot files queued during steps (more than the two staging buffers)
    hold the fields of the step they were taken at, in the context's storage
    type; TAvg over the steps equals the mean of the snapshots."""
    from falm_b200 import api
    from falm_b200.driver import Simulation
    case = small_cases()["channel"]
    sim = Simulation(case, precision)
    ctx = sim.ctx
    uavg, pavg = ctx.field(3), ctx.field(1)
    kept = []
    for q in range(5):
        sim.step()
        ctx.tavg(uavg, sim.u, q + 1)
        ctx.tavg(pavg, sim.p, q + 1)
        ctx.write_vector_file(tmp_path / f"s{q}.bin", [sim.u, sim.p], sim.it, sim.t())
        kept.append((host(sim.u), host(sim.p)))
    ctx.io_wait()
    g = case.grid
    for q in range(5):
        hd, data = api.read_vector_file(tmp_path / f"s{q}.bin")
        assert (hd["imax"], hd["jmax"], hd["kmax"], hd["ncol"], hd["gc"], hd["step"]) == (g.sx, g.sy, g.sz, 4, g.gc, q + 1)
        assert hd["time"] == (q + 1) * case.dt and hd["dsize"] == (8 if precision == "fp64" else 4)
        np.testing.assert_array_equal(data[:3].ravel().astype(np.float64), kept[q][0])
        np.testing.assert_array_equal(data[3].ravel().astype(np.float64), kept[q][1])
    tol = 1e-14 if precision == "fp64" else 1e-6
    assert rel_l2(host(uavg), np.mean([k[0] for k in kept], axis=0)) < tol
    assert rel_l2(host(pavg), np.mean([k[1] for k in kept], axis=0)) < tol
    sim.close()


def test_driver_output_schedule(lib_built, tmp_path):
    """Simulation.enable_output: the files of FalmSolver's schedule (every second
    step from step 2 to 6, averaging over steps 3..5) and the index entries."""
    import json
    from falm_b200 import api
    from falm_b200.driver import Simulation
    case = small_cases()["channel"]
    sim = Simulation(case, "mixed")
    sim.enable_output(tmp_path / "o", 2, start=2, end=6, tavg_start=3, tavg_end=5, as_fp64=True)
    for _ in range(7):
        sim.step()
    sim.finish_output()
    names = sorted(x for x in __import__("os").listdir(tmp_path) if x.startswith("o_"))
    assert names == ["o_000000_0000000002", "o_000000_0000000004", "o_000000_0000000006", "o_tavg_000000_0000000004"]
    idx = json.loads((tmp_path / "o.json").read_text())
    assert [(s["step"], s.get("timeAvg", 0)) for s in idx["outputSteps"]] == [(2, 0), (4, 1), (6, 0)]
    assert idx["dataType"] == "float64"
    hd, _ = api.read_vector_file(tmp_path / "o_000000_0000000006")
    assert hd["dsize"] == 8 and hd["step"] == 6
    sim.close()


def test_step_mixed_odd_width(oracle, lib_built):
    """Mixed precision on an odd interior width (row kernels throughout) against
    the FP64 oracle."""
    case = small_cases()["odd"]
    case.tol = 1e-8
    ref, rs = run_oracle(oracle, case, 10)
    got, gs, _ = run_gpu(case, 10, precision="mixed")
    err = compare(case, got, ref)
    assert err["u"] < 2e-4 and err["uu"] < 2e-4, err
    for a, b in zip(gs, rs):
        assert a["torque"][0] == pytest.approx(b["torque"][0], rel=5e-3)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_reports_non_finite_input(lib_built, precision):
    """A NaN in the velocity reaches the solver's FP64 reductions: falm_step
    stops with FALM_ERR_NAN (3) instead of continuing, and the same context then
    steps normally from a clean state."""
    from falm_b200._lib import FalmError
    case = small_cases()["channel"]
    g = case.grid
    ctx = make_ctx(case, precision)
    st0 = cases.initial_state(case)
    bad = st0["u"].copy()
    bad[g.gc + 5 + g.sx * ((g.gc + 4) + g.sy * (g.gc + 3))] = np.nan
    u, uu, p, nut = dev(ctx, bad), ctx.field(3), ctx.field(1), ctx.field(1)
    ctx.utouu(u, uu)
    ctx.sgs(u, nut)
    with pytest.raises(FalmError) as e:
        ctx.step(u, uu, p, nut, None, case.dt, case.dt)
    assert e.value.code == 3
    u, uu, p, nut = dev(ctx, st0["u"]), ctx.field(3), ctx.field(1), ctx.field(1)
    ctx.utouu(u, uu)
    ctx.sgs(u, nut)
    s = ctx.step(u, uu, p, nut, None, case.dt, case.dt)
    assert s["status"] == 0 and np.isfinite(host(u)).all()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bounded_wait_gives_up_and_context_recovers(oracle, lib_built, precision):
    """Failure detection of the bounded device waits.  falm_debug_arm_wait_probe
    makes the next step start with a wait on an mbarrier that no copy ever
    completes (the bounded wait of the plane streams, limited to 20000 clock64
    cycles).  The wait gives up, the step finishes its other kernels, reads the
    device error word and returns FALM_ERR_TIMEOUT instead of hanging; the
    error word is then clear, and the same context runs the following steps
    correctly (FP64: equal to the oracle at 1e-10 in fixed-iteration mode;
    mixed: velocities within 2e-4 of the FP64 oracle in convergence mode)."""
    import ctypes
    import torch
    from falm_b200 import _lib as L
    case = small_cases()["wide"]
    fixed = precision == "fp64"   # mixed: the drivers' convergence mode (outer FP64 refinement needs a tolerance)
    if not fixed:
        case.tol = 1e-8
    ctx = make_ctx(case, precision)
    if fixed:
        ctx.eq_init(6, 0.0, case.pc, case.pc_maxit, case.pc_relax)
    st0 = cases.initial_state(case)
    u, uu, p, nut = dev(ctx, st0["u"]), ctx.field(3), ctx.field(1), ctx.field(1)
    ctx.utouu(u, uu)
    ctx.sgs(u, nut)
    assert ctx.lib.falm_debug_arm_wait_probe(ctx.h, ctypes.c_longlong(0)) == L.FALM_ERR_ARG
    assert ctx.lib.falm_debug_arm_wait_probe(ctx.h, ctypes.c_longlong(20000)) == L.FALM_OK
    with pytest.raises(L.FalmError) as e:
        ctx.step(u, uu, p, nut, None, case.dt, case.dt)
    assert e.value.code == L.FALM_ERR_TIMEOUT
    assert "bounded wait" in str(e.value)
    # the context is usable: start again from the initial state
    u.copy_(dev(ctx, st0["u"]))
    p.zero_()
    ctx.utouu(u, uu)
    ctx.sgs(u, nut)
    gs = [ctx.step(u, uu, p, nut, None, case.dt, (it + 1) * case.dt) for it in range(3)]
    torch.cuda.synchronize()
    ref, rs = run_oracle(oracle, case, 3, maxit=6 if fixed else None, tol=0.0 if fixed else None)
    err = compare(case, {"u": host(u), "uu": host(uu), "p": host(p), "nut": host(nut)}, ref)
    if fixed:
        for k, v in err.items():
            assert v < 1e-10, (k, v, err)
        for a, b in zip(gs, rs):
            assert a["it"] == b["it"]
    else:
        assert err["u"] < 2e-4 and err["uu"] < 2e-4, err
        for a, b in zip(gs, rs):
            assert a["torque"][0] == pytest.approx(b["torque"][0], rel=5e-3)
    ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_from_saved_state(lib_built, tmp_path, precision):
    """Checkpoint/resume: the step state saved after 3 steps (the snapshot
    format, falm_io_write_vector_file) and read back into a new simulation
    (falm_io_read_vector_file) continues the run exactly -- 3 + 2 steps equal 5
    uninterrupted steps bit for bit; a truncated or mismatched file is refused
    with FALM_ERR_ARG and leaves the fields unchanged."""
    from falm_b200 import _lib as L
    from falm_b200.driver import Simulation
    case = small_cases()["channel"]
    ref = Simulation(case, precision)
    for _ in range(5):
        ref.step()
    a = Simulation(case, precision)
    for _ in range(3):
        a.step()
    a.save_state(tmp_path / "s3")
    b = Simulation(case, precision)
    b.load_state(tmp_path / "s3")
    assert b.it == 3
    for _ in range(2):
        b.step()
    for k in ("u", "uu", "p", "nut"):
        assert np.array_equal(getattr(b, k).cpu().numpy(), getattr(ref, k).cpu().numpy()), k
    raw = (tmp_path / "s3").read_bytes()
    (tmp_path / "cut").write_bytes(raw[:len(raw) - 8])
    (tmp_path / "long").write_bytes(raw + b"\0" * 8)
    (tmp_path / "head").write_bytes(raw[:40])
    before = b.u.cpu().numpy().copy()
    for name in ("cut", "long", "head"):
        with pytest.raises(L.FalmError) as e:
            b.load_state(tmp_path / name)
        assert e.value.code == L.FALM_ERR_ARG
    assert np.array_equal(b.u.cpu().numpy(), before)
    b.step()
    for s in (ref, a, b):
        s.ctx.close()


def test_inconsistent_rhs_ends_in_a_status(lib_built):
    """A right-hand side outside the range of the singular all-Neumann cavity
    operator (a constant: the system has no solution) makes BiCGStab stall or
    break down: the solve ends in a status (FALM_ERR_MAXIT, FALM_ERR_BREAKDOWN,
    or FALM_ERR_NAN for a non-finite alpha/omega, after which no kernel updates
    the iterate) with a finite iterate, never a trap or a hang, and the
    context then solves a consistent system normally."""
    from falm_b200.api import _ptr
    import ctypes
    case = cases.cavity(16)
    g = case.grid
    ctx = make_ctx(case)
    ctx.eq_init(200, 1e-12, case.pc, case.pc_maxit, case.pc_relax)
    b = np.zeros((g.sz, g.sy, g.sx))
    gc = g.gc
    b[gc:-gc, gc:-gc, gc:-gc] = 1.0
    x, r = ctx.field(1), ctx.field(1)
    it, err = ctypes.c_int(), ctypes.c_double()
    rc = ctx.lib.falm_eq_solve(ctx.h, _ptr(x), _ptr(dev(ctx, b.reshape(-1))), _ptr(r), ctx.stream(), ctypes.byref(it),
                               ctypes.byref(err))
    assert rc in (3, 4, 5), rc
    assert np.isfinite(host(x)).all()
    # a consistent right-hand side (zero mean) on the same context
    bc = b.copy()
    bc[gc:-gc, gc:-gc, gc:-gc] = np.random.default_rng(2).standard_normal((g.sz - 2 * gc, g.sy - 2 * gc, g.sx - 2 * gc))
    bc[gc:-gc, gc:-gc, gc:-gc] -= bc[gc:-gc, gc:-gc, gc:-gc].mean()
    ctx.eq_init(200, 1e-10, case.pc, case.pc_maxit, case.pc_relax)
    x2 = ctx.field(1)
    its, errv, rc2 = ctx.solve(x2, dev(ctx, bc.reshape(-1)), r)
    assert rc2 == 0 and errv <= 1e-10 and np.isfinite(host(x2)).all()
    ctx.close()
