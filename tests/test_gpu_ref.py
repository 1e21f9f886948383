"""Parity with the reference's OWN CUDA implementation (oracle/_ref/libfalmref.so,
compiled from the reference's sources by oracle/Makefile) on identical inputs:

  * pins the CPU oracle operator by operator and over whole steps, and
  * checks the B200 FP64 path against the reference's step: relative L2 <= 1e-10
    after 10 steps (the difference comes from reduction order and contraction).

Skipped when the prebuilt reference library is absent."""
import os
import tempfile

import numpy as np
import pytest

from falm_b200 import cases
from tests.helpers import faces, interior, random_state, rel_l2
from tests.test_gpu_step import compare, run_gpu, run_oracle

pytestmark = pytest.mark.gpu

REF_SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libfalmref.so")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built (needs the reference sources)")


def ref_for(case, **kw):
    from oracle.oracle import CaseStruct, RefStep
    cs = CaseStruct(case, use_inflow=False, **kw)
    return RefStep(cs, tempfile.mkdtemp(prefix="falmref_")), cs


def ref_run(case, steps, **kw):
    ref, cs = ref_for(case, **kw)
    st = cases.initial_state(case)
    ref.set("U", st["u"])
    ref.op("UTOUU")
    ref.op("SGS")
    stats = [ref.step((it + 1) * case.dt) for it in range(steps)]
    out = {k: ref.get(n) for k, n in (("u", "U"), ("uu", "UU"), ("p", "P"), ("nut", "NUT"))}
    ref.close()
    return out, stats


def uniform_inflow_cases():
    ch = cases.small_channel(32, 20, 20, intensity=0.0)     # the reference has uniform inflow only
    cav = cases.cavity(16)
    cav.tol = 1e-10
    return {"channel": ch, "cavity": cav}


@needs_ref
def test_oracle_ops_match_reference(oracle):
    import ctypes
    from oracle.oracle import CaseStruct, _p
    case = cases.small_channel(24, 16, 16, intensity=0.0)
    ref, cs = ref_for(case)
    m = oracle.setup(cs)
    g = case.grid
    assert ref.maxdiag() == pytest.approx(m["maxdiag"], rel=1e-15)
    np.testing.assert_allclose(interior(ref.get("A"), g, 7), interior(m["A"], g, 7), rtol=1e-15, atol=1e-16)
    st = random_state(case, seed=3)
    c = ctypes.byref(cs.c)
    # pseudo-velocity
    for k in ("U", "UU", "NUT", "FF"):
        ref.set(k, st[k.lower()])
    ref.op("PSEUDO_U")
    ua = np.zeros(3 * g.n)
    oracle.L.oracle_pseudo_u(c, _p(st["u"]), _p(st["u"]), _p(st["uu"]), _p(ua), _p(st["nut"]), _p(m["kx"]), _p(m["g"]),
                             _p(m["ja"]), _p(st["ff"]))
    assert rel_l2(interior(ref.get("U"), g, 3), interior(ua, g, 3)) < 1e-13
    # UtoUU
    ref.set("U", st["u"])
    ref.op("UTOUU")
    uu = st["uu"].copy()
    oracle.L.oracle_utouu(c, _p(st["u"]), _p(uu), _p(m["kx"]), _p(m["ja"]))
    assert rel_l2(faces(ref.get("UU"), g), faces(uu, g)) < 1e-14
    # RHS
    ref.op("RHS")
    rhs = np.zeros(g.n)
    oracle.L.oracle_poisson_rhs(c, _p(uu), _p(rhs), _p(m["ja"]), m["maxdiag"])
    assert rel_l2(interior(ref.get("RHS"), g), interior(rhs, g)) < 1e-13
    # projection, pbc, ubc, SGS
    for k in ("U", "UU", "P"):
        ref.set(k, st[k.lower()])
    ref.op("PBC")
    p = st["p"].copy()
    oracle.L.oracle_pbc(c, _p(p))
    np.testing.assert_array_equal(ref.get("P"), p)
    ref.op("PROJECT")
    u, uu = st["u"].copy(), st["uu"].copy()
    oracle.L.oracle_project_p(c, _p(u), _p(u), _p(uu), _p(uu), _p(p), _p(m["kx"]), _p(m["g"]))
    assert rel_l2(interior(ref.get("U"), g, 3), interior(u, g, 3)) < 1e-14
    assert rel_l2(faces(ref.get("UU"), g), faces(uu, g)) < 1e-14
    uprev = st["u"] + 0.01
    ref.set("UPREV", uprev)
    ref.set("U", st["u"])
    ref.op("UBC", t=0.3)
    u = st["u"].copy()
    oracle.L.oracle_ubc(c, _p(u), _p(uprev), 0.3)
    np.testing.assert_allclose(ref.get("U"), u, rtol=1e-14, atol=1e-16)
    ref.op("SGS")
    nut = np.zeros(g.n)
    oracle.L.oracle_sgs(c, _p(u), _p(nut), _p(m["kx"]), _p(m["ja"]))
    assert rel_l2(interior(ref.get("NUT"), g), interior(nut, g)) < 1e-13
    # ALM (dense Gaussian sum in both)
    ref.set("U", st["u"])
    s = ref.op("ALM", t=0.41)
    ff = np.zeros(3 * g.n)
    out = oracle.alm(cs, st["u"], ff, 0.41)
    assert s.torque[0] == pytest.approx(out["torque"][0], rel=1e-12)
    assert s.thrust[0] == pytest.approx(out["thrust"][0], rel=1e-12)
    assert rel_l2(interior(ref.get("FF"), g, 3), interior(ff, g, 3)) < 1e-12
    ref.close()


@needs_ref
@pytest.mark.parametrize("name", ["channel", "cavity"])
def test_oracle_step_matches_reference(oracle, name):
    case = uniform_inflow_cases()[name]
    ref, rs = ref_run(case, 10, maxit=6, tol=0.0)
    got, gs = run_oracle(oracle, case, 10, maxit=6, tol=0.0)
    err = compare(case, got, ref)
    for k, v in err.items():
        assert v < 1e-10, (k, v, err)


@needs_ref
@pytest.mark.parametrize("name", ["channel", "cavity"])
def test_b200_step_matches_reference_fixed_iterations(lib_built, name):
    """north-star parity: FP64 B200 step vs the reference's own step, 10 steps,
    relative L2 <= 1e-10 on every field.  Fixed-iteration mode (tol 0, maxit 6)
    removes the stopping rule, so the only differences are rounding order."""
    case = uniform_inflow_cases()[name]
    ref, rs = ref_run(case, 10, maxit=6, tol=0.0)
    got, gs, _ = run_gpu(case, 10, maxit=6, tol=0.0)
    for a, b in zip(gs, rs):
        assert a["it"] == b["it"]
        for x, y in zip(a["torque"] + a["thrust"], b["torque"] + b["thrust"]):
            assert x == pytest.approx(y, rel=1e-10)
    err = compare(case, got, ref)
    for k, v in err.items():
        assert v < 1e-10, (k, v, err)


@needs_ref
@pytest.mark.parametrize("name", ["channel", "cavity"])
def test_b200_step_matches_reference_converged(lib_built, oracle, name):
    """Convergence mode (the drivers' tol): iteration counts within +-1.  A
    BiCGStab iterate stopped at a residual tolerance is determined only to that
    tolerance and Krylov iterations amplify rounding differences, so the pressure
    is compared at 1e-6 and the velocities at 1e-9; the oracle shows the same
    spread against the reference, which is checked here too."""
    case = uniform_inflow_cases()[name]
    ref, rs = ref_run(case, 10)
    got, gs, _ = run_gpu(case, 10)
    orc, os_ = run_oracle(oracle, case, 10)
    for a, b in zip(gs, rs):
        assert abs(a["it"] - b["it"]) <= 1
        for x, y in zip(a["torque"] + a["thrust"], b["torque"] + b["thrust"]):
            assert x == pytest.approx(y, rel=1e-8)
    for other in (got, orc):
        err = compare(case, other, ref)
        assert err["u"] < 1e-9 and err["uu"] < 1e-9 and err["nut"] < 1e-9, err
        assert err["p"] < 1e-6, err


@needs_ref
@pytest.mark.parametrize("ls,relax", [("Jacobi", 1.0), ("SOR", 1.3)])
def test_plain_solvers_match_reference(oracle, lib_built, ls, relax):
    """FalmEq::Jacobi / FalmEq::SOR: the reference's own solver, the oracle's
    restatement and the B200 solver in fixed-iteration mode (tol 0, maxit 6) on
    the same operator, right-hand side and initial guess."""
    from oracle.oracle import CaseStruct
    from tests.helpers import dev, host, make_ctx
    case = uniform_inflow_cases()["channel"]
    g = case.grid
    rng = np.random.default_rng(3)
    b = np.zeros(g.n)
    interior(b, g)[...] = rng.standard_normal(interior(b, g).shape)
    x0 = 0.1 * rng.standard_normal(g.n)
    ref, _ = ref_for(case)
    ref.set("RHS", b)
    ref.set("P", x0)
    it_r, err_r = ref.plain_solve(ls, relax, 6, 0.0)
    xr, rr = ref.get("P"), ref.get("RES")
    ref.close()
    cs = CaseStruct(case, use_inflow=False, maxit=6, tol=0.0)
    m = oracle.setup(cs)
    xo, ro = x0.copy(), np.zeros(g.n)
    it_o, err_o = oracle.plain_solve(cs, ls, relax, m["A"], xo, b, ro)
    ctx = make_ctx(case)
    ctx.eq_init(6, 0.0, case.pc, case.pc_maxit, case.pc_relax, ls=ls, relax=relax)
    xd, bd, rd = dev(ctx, x0), dev(ctx, b), ctx.field(1)
    it, err, rc = ctx.solve(xd, bd, rd)
    assert it_r == it_o == it == 6
    assert rel_l2(interior(xo, g), interior(xr, g)) < 1e-12
    assert rel_l2(interior(host(xd), g), interior(xr, g)) < 1e-12
    assert rel_l2(interior(host(rd), g), interior(rr, g)) < 1e-10
    assert err_o == pytest.approx(err_r, rel=1e-10) and err == pytest.approx(err_r, rel=1e-10)


@needs_ref
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_output_files_match_reference(lib_built, tmp_path, precision):
    """FalmIO byte for byte against the reference's own writers on the same
    state: the drivers' u + p vector file (an FP32 context cast to FP64 on the
    device, from a state exactly representable in FP32), the index file and the
    control-volume file of a stretched grid."""
    from falm_b200 import api
    from tests.helpers import dev, make_ctx
    case = cases.Case("stretched", cases.stretched_grid(20, 14, 12, 0.1), 0, Re=500.0, dt=0.01, tol=1e-10)
    g = case.grid
    st = random_state(case, seed=31)
    u = st["u"].astype(np.float32).astype(np.float64)
    p = st["p"].astype(np.float32).astype(np.float64)
    ref, _ = ref_for(case)
    ref.set("U", u)
    ref.set("P", p)
    ref.write_uvwp(tmp_path / "ref.bin", 1234, 18.51)
    snaps = [(100, 1.5, False), (200, 0.01 * 200, True), (300, 0.1 + 0.2, True), (7, 1e-05, False), (8, 2.5e15, False)]
    ref.write_index(tmp_path / "ref.json", snaps)
    ref.write_cv(tmp_path / "ref.cv")
    ref.close()
    ctx = make_ctx(case, precision)
    ud, pd = dev(ctx, u), dev(ctx, p)
    ctx.write_vector_file(tmp_path / "b200.bin", [ud, pd], 1234, 18.51, as_fp64=True)
    ctx.io_wait()
    api.write_index_file(tmp_path / "b200.json", g.interior, g.gc, snaps)
    ctx.write_cv_file(tmp_path / "b200.cv")
    for name in ("bin", "json", "cv"):
        assert (tmp_path / f"b200.{name}").read_bytes() == (tmp_path / f"ref.{name}").read_bytes(), name
    dims, x, hx, y, hy, z, hz = api.read_cv_file(tmp_path / "ref.cv")
    assert dims == (g.sx, g.sy, g.sz, g.gc)
    for a, b in ((x, g.x), (hx, g.hx), (y, g.y), (hy, g.hy), (z, g.z), (hz, g.hz)):
        np.testing.assert_allclose(a, b, rtol=1e-14, atol=0)


# ---------------------------------------------------------------- the configurations' own sizes
@needs_ref
def test_b200_cavity_64_100_steps_matches_reference(oracle, lib_built):
    """The lid-driven cavity configuration at its own size and length (64^3,
    Re 1000, dt 1e-3, Upwind3, Smagorinsky Cs 0.1, PBiCGStab + RB-SOR x2): the
    FP64 B200 step against the reference's own step over all 100 steps.
      * fixed-iteration mode (tol 0, maxit 6): relative L2 <= 1e-10 on every field;
      * convergence mode (tol 1e-8, err = ||r||/N): BiCGStab iteration counts
        within +-1 at every step.  Each step's pressure is determined only to
        the stopping tolerance, and over 100 steps the runs drift apart by the
        accumulated solver truncation: the CPU oracle, a plain restatement,
        drifts from the reference by the same order.  Bound: velocities 1e-7,
        pressure 1e-5, and at most 10x the oracle's own distance (floor 1e-9)."""
    case = cases.cavity(64)
    ref, rs = ref_run(case, 100, maxit=6, tol=0.0)
    got, gs, _ = run_gpu(case, 100, maxit=6, tol=0.0)
    assert [a["it"] for a in gs] == [b["it"] for b in rs]
    err = compare(case, got, ref)
    for k, v in err.items():
        assert v < 1e-10, (k, v, err)
    ref, rs = ref_run(case, 100)
    got, gs, _ = run_gpu(case, 100)
    orc, os_ = run_oracle(oracle, case, 100)
    for a, b in zip(gs, rs):
        assert abs(a["it"] - b["it"]) <= 1, ([x["it"] for x in gs], [x["it"] for x in rs])
        assert a["err"] <= case.tol
    err = compare(case, got, ref)
    spread = compare(case, orc, ref)
    for k in ("u", "uu", "nut"):
        assert err[k] < 1e-7 and err[k] < max(1e-9, 10 * spread[k]), (k, err, spread)
    assert err["p"] < 1e-5 and err["p"] < max(1e-9, 10 * spread["p"]), (err, spread)


@needs_ref
def test_b200_channel_256_rotor_matches_reference(lib_built):
    """The 256x128x128 channel with the full-size rotor (R = 20 cells, TSR 7,
    3 x 32 actuator points, Gaussian width 2h; uniform inflow, which is the
    reference's only inlet): 10 FP64 steps in fixed-iteration mode (tol 0,
    maxit 6) against the reference's own step.  This size runs every multi-chunk
    plane stream, the clamped boxes of a 260-wide row and the force-box ALM
    projection at its real extent; the reference projects the AP forces densely
    over the whole grid.  Relative L2 <= 1e-10 on u, uu, p, nut; torque and
    thrust at every step within 1e-10."""
    case = cases.channel(256, 128, 128, intensity=0.0)
    ref, rs = ref_run(case, 10, maxit=6, tol=0.0)
    got, gs, _ = run_gpu(case, 10, maxit=6, tol=0.0)
    for a, b in zip(gs, rs):
        assert a["it"] == b["it"]
        for x, y in zip(a["torque"] + a["thrust"], b["torque"] + b["thrust"]):
            assert x == pytest.approx(y, rel=1e-10)
    err = compare(case, got, ref)
    for k, v in err.items():
        assert v < 1e-10, (k, v, err)


def variant_cases():
    """the reference's other advection schemes and the Jacobi preconditioner
    (src/FalmCFDScheme.h:8-132, src/FalmEq.cpp:129-171), each on the channel and
    the cavity, and the scheme-free step (no SGS model)"""
    out = {}
    for name, mk in (("channel", lambda: cases.small_channel(32, 20, 20, intensity=0.0)),
                     ("cavity", lambda: cases.cavity(16))):
        for adv in ("Upwind1", "QUICK", "UTOPIA", "KK"):
            c = mk()
            c.adv = adv
            out[f"{name}-{adv}"] = c
        c = mk()
        c.pc, c.pc_maxit, c.pc_relax = "Jacobi", 2, 1.0
        out[f"{name}-JacobiPC"] = c
        c = mk()
        c.adv, c.sgs = "KK", "Empty"
        out[f"{name}-KK-noSGS"] = c
    return out


@needs_ref
def test_csm_operator_matches_reference(oracle, lib_built):
    """The CSM eddy viscosity (src/dev/FalmCFDDevCall.cu:478-555) of the
    reference's own FalmCFD::SGS, of the oracle and of the B200 kernel on the
    same random velocity field.  The reference takes sqrt(fcs^3) of the signed
    coefficient fcs = Q/E (its |fcs| is computed and not used, :548-549), so
    every cell with Q < 0 gets NaN there; all three give NaN at exactly the same
    cells and agree to 1e-13 elsewhere.  (A time step with CSM meets such cells
    at once in any sheared flow: the B200 step then stops with FALM_ERR_NAN,
    where the reference carries the NaN on.)"""
    import ctypes
    from oracle.oracle import _p
    from tests.helpers import dev, host, make_ctx
    for name, case in (("channel", cases.small_channel(32, 20, 20, intensity=0.0)), ("cavity", cases.cavity(16))):
        case.sgs = "CSM"
        g = case.grid
        ref, cs = ref_for(case)
        m = oracle.setup(cs)
        st = random_state(case, seed=11)
        ref.set("U", st["u"])
        ref.op("SGS")
        want = interior(ref.get("NUT"), g)
        ref.close()
        nut_o = np.zeros(g.n)
        oracle.L.oracle_sgs(ctypes.byref(cs.c), _p(st["u"]), _p(nut_o), _p(m["kx"]), _p(m["ja"]))
        ctx = make_ctx(case)
        nut_d = ctx.field(1)
        ctx.sgs(dev(ctx, st["u"]), nut_d)
        got = interior(host(nut_d), g)
        orc = interior(nut_o, g)
        ctx.close()
        nan = np.isnan(want)
        assert 0 < nan.sum() < nan.size, name
        for other in (got, orc):
            assert np.array_equal(np.isnan(other), nan), name
            assert rel_l2(other[~nan], want[~nan]) < 1e-13, name


@needs_ref
@pytest.mark.parametrize("name", sorted(variant_cases()))
def test_variants_match_reference(oracle, lib_built, name):
    """Every variant through the reference's own FalmCFD / FalmEq (oracle/_ref):
    the CPU oracle's restatement and the FP64 B200 step both within 1e-10
    relative L2 of it after 10 steps in fixed-iteration mode (tol 0, maxit 6),
    with equal BiCGStab iteration counts and equal rotor torque and thrust."""
    case = variant_cases()[name]
    ref, rs = ref_run(case, 10, maxit=6, tol=0.0)
    orc, os_ = run_oracle(oracle, case, 10, maxit=6, tol=0.0)
    got, gs, _ = run_gpu(case, 10, maxit=6, tol=0.0)
    for other, st in ((orc, os_), (got, gs)):
        err = compare(case, other, ref)
        for k, v in err.items():
            assert v < 1e-10, (k, v, err)
        for a, b in zip(st, rs):
            assert a["it"] == b["it"]
            for x, y in zip(a["torque"] + a["thrust"], b["torque"] + b["thrust"]):
                assert x == pytest.approx(y, rel=1e-10)
