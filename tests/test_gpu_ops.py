"""Per-operator parity of the CUDA path (through the C ABI) with the CPU oracle,
FP64, on seeded random inputs.  The tolerance is relative L2 <= 1e-12: both sides
evaluate the same expressions and differ by FMA contraction only."""
import ctypes

import numpy as np
import pytest

from falm_b200 import cases
from tests.helpers import dev, faces, host, interior, make_ctx, random_state, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _setup(oracle, case):
    from oracle.oracle import CaseStruct
    cs = CaseStruct(case)
    m = oracle.setup(cs)
    return cs, m


def _p(a):
    from oracle.oracle import _p as pp
    return pp(a)


CASES = {
    "channel": lambda: cases.small_channel(24, 16, 12, intensity=0.05).with_inflow(nb=8),
    "cavity": lambda: cases.cavity(12),
    "stretched": lambda: cases.Case("stretched", cases.stretched_grid(20, 14, 12, 0.1), 0, Re=500.0, dt=0.01, tol=1e-10),
}


@pytest.fixture(params=list(CASES))
def case(request):
    return CASES[request.param]()


@pytest.mark.parametrize("adv", ["Upwind3", "Upwind1", "QUICK", "UTOPIA", "KK"])
def test_pseudo_u(oracle, lib_built, adv):
    case = CASES["stretched"]()
    case.adv = adv
    cs, m = _setup(oracle, case)
    st = random_state(case)
    ua = np.zeros_like(st["u"])
    oracle.L.oracle_pseudo_u(ctypes.byref(cs.c), _p(st["u"]), _p(st["u"]), _p(st["uu"]), _p(ua), _p(st["nut"]),
                             _p(m["kx"]), _p(m["g"]), _p(m["ja"]), _p(st["ff"]))
    ctx = make_ctx(case)
    u, uu, nut, ff = dev(ctx, st["u"]), dev(ctx, st["uu"]), dev(ctx, st["nut"]), dev(ctx, st["ff"])
    ua_d = ctx.field(3)
    ctx.pseudo_u(u, u, uu, ua_d, nut, ff, case.dt)
    assert rel_l2(interior(host(ua_d), case.grid, 3), interior(ua, case.grid, 3)) < TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("shape", [(20, 14, 12), (64, 24, 70), (36, 9, 5), (21, 10, 7), (67, 13, 9)])
def test_pseudo_u_tma_matches_row_kernel(lib_built, monkeypatch, precision, shape):
    """The TMA-streamed 2.5D kernels and the plain row kernel agree (partial
    tiles in x/y, z chunks, ALM force evaluated in-kernel). An odd interior
    width takes the one-cell kernel in FP32 too (the x-pair kernel needs every
    pair inside the interior or outside it)."""
    case = cases.small_channel(*shape, intensity=0.0)
    st = random_state(case, seed=12)
    outs = []
    for no_tma in ("1", "0"):
        monkeypatch.setenv("FALM_B200_NO_TMA", no_tma)
        ctx = make_ctx(case, precision)
        u, uu, nut = dev(ctx, st["u"]), dev(ctx, st["uu"]), dev(ctx, st["nut"])
        ctx.alm_run(u, None, 0.2)
        ua = ctx.field(3)
        ctx.pseudo_u(u, u, uu, ua, nut, None, case.dt)
        outs.append(interior(host(ua), case.grid, 3))
    tol = 1e-14 if precision == "fp64" else 1e-6
    assert rel_l2(outs[1], outs[0]) < tol


@pytest.mark.parametrize("adv", ["Upwind3", "UTOPIA", "KK"])
@pytest.mark.parametrize("shape", [(20, 14, 12), (64, 24, 70), (36, 9, 5), (96, 20, 16)])
def test_pseudo_u_pair_kernel_matches_one_cell_kernel(lib_built, monkeypatch, adv, shape):
    """FP32: the x-pair pseudo-velocity kernel (two cells per thread) and the
    one-cell-per-thread kernel evaluate the same update (partial tiles, z chunks,
    the ALM force from the force boxes); they may differ in rounding only."""
    case = cases.small_channel(*shape, intensity=0.0)
    case.adv = adv
    st = random_state(case, seed=5)
    outs = []
    for v1 in ("1", "0"):
        monkeypatch.setenv("FALM_B200_PU_V1", v1)
        ctx = make_ctx(case, "mixed")
        u, uu, nut = dev(ctx, st["u"]), dev(ctx, st["uu"]), dev(ctx, st["nut"])
        ctx.alm_run(u, None, 0.2)
        ua = ctx.field(3)
        ctx.pseudo_u(u, u, uu, ua, nut, None, case.dt)
        outs.append(interior(host(ua), case.grid, 3))
    assert np.isfinite(outs[1]).all()
    assert rel_l2(outs[1], outs[0]) < 1e-6
    # the update itself (ua - u) agrees closely too
    u0 = interior(st["u"].astype(np.float32).astype(np.float64), case.grid, 3)
    assert rel_l2(outs[1] - u0, outs[0] - u0) < 1e-4


def test_pseudo_u_rejects_alias(lib_built):
    case = CASES["cavity"]()
    ctx = make_ctx(case)
    u = ctx.field(3)
    with pytest.raises(Exception):
        ctx.pseudo_u(u, u, ctx.field(3), u, ctx.field(1), ctx.field(3), case.dt)


def test_utouu_rhs_project_sgs_div(oracle, lib_built, case):
    cs, m = _setup(oracle, case)
    g = case.grid
    st = random_state(case, seed=11)
    c = ctypes.byref(cs.c)
    ctx = make_ctx(case)
    # UtoUU
    uu_o = st["uu"].copy()
    oracle.L.oracle_utouu(c, _p(st["u"]), _p(uu_o), _p(m["kx"]), _p(m["ja"]))
    u_d, uu_d = dev(ctx, st["u"]), dev(ctx, st["uu"])
    ctx.utouu(u_d, uu_d)
    assert rel_l2(faces(host(uu_d), g), faces(uu_o, g)) < TOL
    # RHS (divergence scaled by 1/(dt maxdiag))
    rhs_o = np.zeros(g.n)
    oracle.L.oracle_poisson_rhs(c, _p(uu_o), _p(rhs_o), _p(m["ja"]), m["maxdiag"])
    rhs_d = ctx.field(1)
    assert ctx.maxdiag == pytest.approx(m["maxdiag"], rel=1e-14)
    ctx.poisson_rhs(uu_d, rhs_d, case.dt, ctx.maxdiag)
    assert rel_l2(interior(host(rhs_d), g), interior(rhs_o, g)) < TOL
    # projection (in place, the drivers' call)
    u_o, uu2_o = st["u"].copy(), st["uu"].copy()
    oracle.L.oracle_project_p(c, _p(u_o), _p(u_o), _p(uu2_o), _p(uu2_o), _p(st["p"]), _p(m["kx"]), _p(m["g"]))
    u_d, uu_d, p_d = dev(ctx, st["u"]), dev(ctx, st["uu"]), dev(ctx, st["p"])
    ctx.project_p(u_d, u_d, uu_d, uu_d, p_d, case.dt)
    assert rel_l2(interior(host(u_d), g, 3), interior(u_o, g, 3)) < TOL
    assert rel_l2(faces(host(uu_d), g), faces(uu2_o, g)) < TOL
    # SGS
    for sgs in ("Smagorinsky", "CSM"):
        case.sgs = sgs
        cs2, _ = _setup(oracle, case)
        nut_o = np.zeros(g.n)
        oracle.L.oracle_sgs(ctypes.byref(cs2.c), _p(st["u"]), _p(nut_o), _p(m["kx"]), _p(m["ja"]))
        ctx.cfd_init(case.Re, case.adv, sgs, case.Cs)
        nut_d = ctx.field(1)
        ctx.sgs(dev(ctx, st["u"]), nut_d)
        got = interior(host(nut_d), g)
        want = interior(nut_o, g)
        if sgs == "CSM":   # sqrt of a negative cube is NaN in both
            assert np.array_equal(np.isnan(got), np.isnan(want))
            got, want = np.nan_to_num(got), np.nan_to_num(want)
        assert rel_l2(got, want) < TOL
    # divergence
    div_o = np.zeros(g.n)
    oracle.L.oracle_divergence(c, _p(st["uu"]), _p(div_o), _p(m["ja"]))
    div_d = ctx.field(1)
    ctx.divergence(dev(ctx, st["uu"]), div_d)
    assert rel_l2(interior(host(div_d), g), interior(div_o, g)) < TOL


def test_operator_mv_dot_res_sor(oracle, lib_built, case):
    cs, m = _setup(oracle, case)
    g = case.grid
    c = ctypes.byref(cs.c)
    rng = np.random.default_rng(5)
    x, b = rng.standard_normal(g.n), rng.standard_normal(g.n)
    ctx = make_ctx(case)
    xd, bd = dev(ctx, x), dev(ctx, b)
    ax_o, ax_d = np.zeros(g.n), ctx.field(1)
    oracle.L.oracle_mv(c, _p(m["A"]), _p(x), _p(ax_o))
    ctx.mv(xd, ax_d)
    assert rel_l2(interior(host(ax_d), g), interior(ax_o, g)) < TOL
    r_o, r_d = np.zeros(g.n), ctx.field(1)
    oracle.L.oracle_res(c, _p(m["A"]), _p(x), _p(b), _p(r_o))
    ctx.res(xd, bd, r_d)
    assert rel_l2(interior(host(r_d), g), interior(r_o, g)) < TOL
    assert ctx.dot(xd, bd) == pytest.approx(oracle.L.oracle_dot(c, _p(x), _p(b)), rel=1e-13)
    assert ctx.normsq(xd) == pytest.approx(oracle.L.oracle_normsq(c, _p(x), 1), rel=1e-13)
    for color in (0, 1):
        xo = x.copy()
        oracle.L.oracle_sor_sweep(c, _p(m["A"]), _p(xo), _p(b), 1.2, color)
        xs = dev(ctx, x)
        ctx.sor_sweep(xs, bd, 1.2, color)
        assert rel_l2(interior(host(xs), g), interior(xo, g)) < TOL
    # the same operator given as an explicit 7-column matrix
    ctx.set_matrix(dev(ctx, m["A"]))
    ax2 = ctx.field(1)
    ctx.mv(xd, ax2)
    assert rel_l2(interior(host(ax2), g), interior(ax_o, g)) < TOL
    assert ctx.maxdiag_of() == pytest.approx(1.0, rel=1e-14)


@pytest.mark.parametrize("pc", ["SOR", "Jacobi"])
def test_pbicgstab_fixed_iterations(oracle, lib_built, pc):
    """FalmEq::PBiCGStab in fixed-iteration mode (tol 0, maxit k): same iterate."""
    case = CASES["channel"]()
    case.pc, case.tol, case.maxit = pc, 0.0, 7
    cs, m = _setup(oracle, case)
    g = case.grid
    rng = np.random.default_rng(9)
    b = np.zeros(g.n)
    interior(b, g)[...] = rng.standard_normal(interior(b, g).shape)
    x0 = 0.1 * rng.standard_normal(g.n)
    xo, ro = x0.copy(), np.zeros(g.n)
    it_o, err_o = oracle.pbicgstab(cs, m["A"], xo, b, ro)
    ctx = make_ctx(case)
    xd, bd, rd = dev(ctx, x0), dev(ctx, b), ctx.field(1)
    it, err, rc = ctx.solve(xd, bd, rd)
    assert it == it_o == 7
    assert err == pytest.approx(err_o, rel=1e-9)
    assert rel_l2(interior(host(xd), g), interior(xo, g)) < 1e-11


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("shape", [(40, 20, 72), (64, 36, 40), (120, 52, 33)])
def test_blocked_sor_tiles_agree(lib_built, monkeypatch, shape, precision):
    """The two temporally blocked red-black SOR kernels (28 x 16 tile with the
    skewed wavefront, 32 x 8 tile with one barrier per half sweep) perform the
    same updates with the same expressions: the solve in fixed-iteration mode
    gives bit-identical iterates in both precisions (partial tiles in x and y,
    several z chunks)."""
    case = cases.small_channel(*shape, intensity=0.0)
    case.pc, case.tol, case.maxit = "SOR", 0.0, 5
    g = case.grid
    rng = np.random.default_rng(4)
    b = np.zeros(g.n)
    interior(b, g)[...] = rng.standard_normal(interior(b, g).shape)
    x0 = 0.1 * rng.standard_normal(g.n)
    outs = []
    for v1 in ("1", "2"):   # the 32 x 8 kernel, then the skewed one
        monkeypatch.setenv("FALM_B200_SOR_V1", v1)
        ctx = make_ctx(case, precision)
        xd, bd, rd = dev(ctx, x0), dev(ctx, b), ctx.field(1)
        ctx.solve(xd, bd, rd)
        outs.append(host(xd))
    assert np.isfinite(outs[1]).all()
    np.testing.assert_array_equal(outs[0], outs[1])


def test_pbicgstab_converged(oracle, lib_built):
    case = CASES["cavity"]()
    case.tol = 1e-10
    cs, m = _setup(oracle, case)
    g = case.grid
    rng = np.random.default_rng(2)
    b = np.zeros(g.n)
    bi = rng.standard_normal(interior(b, g).shape)
    interior(b, g)[...] = bi - bi.mean()     # compatible with the all-Neumann operator
    xo, ro = np.zeros(g.n), np.zeros(g.n)
    it_o, err_o = oracle.pbicgstab(cs, m["A"], xo, b, ro)
    ctx = make_ctx(case)
    xd, rd = ctx.field(1), ctx.field(1)
    it, err, rc = ctx.solve(xd, dev(ctx, b), rd)
    assert abs(it - it_o) <= 1
    assert err <= case.tol
    assert rel_l2(interior(host(xd), g), interior(xo, g)) < 1e-7


@pytest.mark.parametrize("ls", ["Jacobi", "SOR"])
@pytest.mark.parametrize("maxit", [4, 7])
@pytest.mark.parametrize("shape", [(24, 16, 12), (72, 20, 16)])
def test_plain_solvers_fixed_iterations(oracle, lib_built, ls, maxit, shape):
    """FalmEq::Jacobi / FalmEq::SOR (src/FalmEq.cpp:80-127, :173-240) in
    fixed-iteration mode (tol 0): the oracle's iterate, residual and err. An even
    and an odd count end the Jacobi alternation in either buffer; nx = 72 runs
    the SOR half sweeps on the 7-point plane stream."""
    case = cases.small_channel(*shape, intensity=0.05).with_inflow(nb=8)
    case.tol, case.maxit = 0.0, maxit
    cs, m = _setup(oracle, case)
    g = case.grid
    rng = np.random.default_rng(21)
    b = np.zeros(g.n)
    interior(b, g)[...] = rng.standard_normal(interior(b, g).shape)
    x0 = 0.1 * rng.standard_normal(g.n)
    xo, ro = x0.copy(), np.zeros(g.n)
    it_o, err_o = oracle.plain_solve(cs, ls, 1.3, m["A"], xo, b, ro)
    ctx = make_ctx(case)
    ctx.eq_init(maxit, 0.0, case.pc, case.pc_maxit, case.pc_relax, ls=ls, relax=1.3)
    xd, bd, rd = dev(ctx, x0), dev(ctx, b), ctx.field(1)
    it, err, rc = ctx.solve(xd, bd, rd)
    assert it == it_o == maxit and rc == 5          # FALM_ERR_MAXIT: tol 0 is never met
    assert err == pytest.approx(err_o, rel=1e-10)
    assert rel_l2(interior(host(xd), g), interior(xo, g)) < 1e-12
    assert rel_l2(interior(host(rd), g), interior(ro, g)) < 1e-10
    # the ghost cells of x are the caller's
    np.testing.assert_array_equal(host(xd)[:g.sx * g.sy], x0[:g.sx * g.sy])


@pytest.mark.parametrize("ls,relax", [("Jacobi", 1.0), ("SOR", 1.5)])
def test_plain_solvers_converged(oracle, lib_built, ls, relax):
    """Convergence mode: the loop stops at the first iterate with ||r||/N <= tol
    (iteration counts within 1 of the oracle's: about 6800 Jacobi and 1200 SOR
    iterations), FP64 and mixed precision (FP32 iterate, FP64 residual norm).
    The channel's p = 0 outlet makes the operator nonsingular; on the
    all-Neumann cavity plain Jacobi does not converge (its iteration matrix has
    the eigenvalue -1 of the checkerboard mode)."""
    case = cases.small_channel(16, 12, 12, intensity=0.0)
    case.tol, case.maxit = 1e-8, 20000
    cs, m = _setup(oracle, case)
    g = case.grid
    rng = np.random.default_rng(5)
    b = np.zeros(g.n)
    interior(b, g)[...] = rng.standard_normal(interior(b, g).shape)
    xo, ro = np.zeros(g.n), np.zeros(g.n)
    it_o, err_o = oracle.plain_solve(cs, ls, relax, m["A"], xo, b, ro)
    assert err_o <= case.tol and it_o < case.maxit
    ctx = make_ctx(case)
    ctx.eq_init(case.maxit, case.tol, case.pc, case.pc_maxit, case.pc_relax, ls=ls, relax=relax)
    xd, rd = ctx.field(1), ctx.field(1)
    it, err, rc = ctx.solve(xd, dev(ctx, b), rd)
    assert rc == 0 and err <= case.tol and abs(it - it_o) <= 1
    assert rel_l2(interior(host(xd), g), interior(xo, g)) < 1e-8
    ctx32 = make_ctx(case, "mixed")
    ctx32.eq_init(case.maxit, 1e-5, case.pc, case.pc_maxit, case.pc_relax, ls=ls, relax=relax)
    x32, r32 = ctx32.field(1), ctx32.field(1)
    it32, err32, rc32 = ctx32.solve(x32, dev(ctx32, b), r32)
    assert rc32 == 0 and err32 <= 1e-5
    # the FP64 residual of the FP32 iterate, by the oracle, meets the tolerance
    r64, xh = np.zeros(g.n), host(x32)
    oracle.L.oracle_res(ctypes.byref(cs.c), _p(m["A"]), _p(xh), _p(b), _p(r64))
    assert np.sqrt(oracle.L.oracle_normsq(ctypes.byref(cs.c), _p(r64), 1)) / g.n_interior <= 1.01e-5


def test_eq_init_preconditioner_rules(lib_built):
    """A plain solver needs no preconditioner (FALM_LS_EMPTY is accepted);
    PBiCGStab needs SOR or Jacobi."""
    from falm_b200._lib import FalmError
    case = CASES["channel"]()
    ctx = make_ctx(case)
    ctx.eq_init(10, 1e-8, "Empty", 0, 1.0, ls="SOR", relax=1.5)
    ctx.eq_init(10, 1e-8, "Empty", 0, 1.0, ls="Jacobi")
    with pytest.raises(FalmError) as e:
        ctx.eq_init(10, 1e-8, "Empty", 2, 1.0)
    assert e.value.code == 1


def test_step_with_plain_sor_solver(lib_built):
    """A whole step with the plain SOR Poisson solver: the step skips the
    BiCGStab start fused into the face-velocity kernel, runs the solver's
    iterations and gives another pressure than PBiCGStab does."""
    case = CASES["channel"]()
    ctx = make_ctx(case)
    ctx.eq_init(5, 0.0, case.pc, case.pc_maxit, case.pc_relax, ls="SOR", relax=1.2)
    st0 = cases.initial_state(case)
    u, uu, p, nut = dev(ctx, st0["u"]), ctx.field(3), ctx.field(1), ctx.field(1)
    ctx.utouu(u, uu)
    ctx.sgs(u, nut)
    s = ctx.step(u, uu, p, nut, None, case.dt, case.dt)
    assert s["it"] == 5
    # the same step with PBiCGStab gives a different pressure: the solver switch took effect
    ctx2 = make_ctx(case)
    ctx2.eq_init(5, 0.0, case.pc, case.pc_maxit, case.pc_relax)
    u2, uu2, p2, nut2 = dev(ctx2, st0["u"]), ctx2.field(3), ctx2.field(1), ctx2.field(1)
    ctx2.utouu(u2, uu2)
    ctx2.sgs(u2, nut2)
    ctx2.step(u2, uu2, p2, nut2, None, case.dt, case.dt)
    assert rel_l2(host(p), host(p2)) > 1e-6
    assert np.isfinite(host(u)).all()


def test_heat1d_explicit_matrix(lib_built):
    """test/heat1d2.cpp:217 on the GPU through falm_eq_set_matrix"""
    from tests.test_oracle_kat import _box_case, heat1d_system
    shape, A, b, exact = heat1d_system()
    case = _box_case(shape, 2, h=0.01)
    case.maxit, case.tol, case.pc, case.pc_maxit, case.pc_relax = 1000, 1e-9, "SOR", 5, 1.5
    from falm_b200.api import Context
    ctx = Context(case.grid, "fp64")
    ctx.eq_init(case.maxit, case.tol, "SOR", 5, 1.5)
    ctx.set_matrix(dev(ctx, A))
    xd, rd = ctx.field(1), ctx.field(1)
    it, err, rc = ctx.solve(xd, dev(ctx, b), rd)
    assert err <= 1e-9
    assert rel_l2(host(xd), exact) < 1e-7


def test_dot_kat_and_maxdiag(lib_built):
    """test/dot.py:15-30 on the GPU: exact integer interior sums; MaxDiag of the fields"""
    from tests.test_oracle_kat import _box_case
    case = _box_case((12, 12, 12), 1)
    case.grid.gc = 1
    k, j, i = np.meshgrid(np.arange(12), np.arange(12), np.arange(12), indexing="ij")
    a = (300 - (i - 7) ** 2 - (j - 2) ** 2 - (k - 5) ** 2).astype(np.float64).ravel()
    b = (150 - i ** 2 - (j - 1) ** 2 - (k - 1) ** 2).astype(np.float64).ravel()
    inside = ((i > 0) & (i < 11) & (j > 0) & (j < 11) & (k > 0) & (k < 11)).ravel()
    from falm_b200.api import Context
    # gc = 1 is below the library's minimum of 2: embed the 12^3 box in a 14^3 one
    big = _box_case((14, 14, 14), 2)
    ctx = Context(big.grid, "fp64")
    A = np.zeros((14, 14, 14)); A[1:13, 1:13, 1:13] = a.reshape(12, 12, 12)
    B = np.zeros((14, 14, 14)); B[1:13, 1:13, 1:13] = b.reshape(12, 12, 12)
    assert ctx.dot(dev(ctx, A.ravel()), dev(ctx, B.ravel())) == float(np.sum((a * b)[inside]))
    assert ctx.normsq(dev(ctx, A.ravel())) == float(np.sum((a * a)[inside]))
    M = np.zeros(7 * 14 ** 3); M[:14 ** 3] = A.ravel()
    ctx.set_matrix(dev(ctx, M))
    assert ctx.maxdiag_of() == float(np.abs(a[inside]).max())


def test_boundary_conditions(oracle, lib_built, case):
    cs, m = _setup(oracle, case)
    g = case.grid
    c = ctypes.byref(cs.c)
    st = random_state(case, seed=4)
    uprev = st["u"] + 0.01
    t = 0.37
    ctx = make_ctx(case)
    u_o = st["u"].copy()
    oracle.L.oracle_ubc(c, _p(u_o), _p(uprev), t)
    u_d = dev(ctx, st["u"])
    ctx.ubc(u_d, dev(ctx, uprev), case.dt, t)
    # every guide cell the reference writes (faces, not edges/corners) must match exactly
    np.testing.assert_allclose(host(u_d), u_o, rtol=1e-13, atol=1e-15)
    p_o = st["p"].copy()
    oracle.L.oracle_pbc(c, _p(p_o))
    p_d = dev(ctx, st["p"])
    ctx.pbc(p_d)
    np.testing.assert_array_equal(host(p_d), p_o)
    uu_o = st["uu"].copy()
    oracle.L.oracle_uubc(c, _p(uu_o))
    uu_d = dev(ctx, st["uu"])
    ctx.uubc(uu_d)
    np.testing.assert_array_equal(host(uu_d), uu_o)


def test_alm_forces_and_projection(oracle, lib_built):
    case = cases.small_channel(40, 28, 28, intensity=0.05)
    cs, m = _setup(oracle, case)
    g = case.grid
    st = random_state(case, seed=21, amp=0.05)
    for t in (0.0, 0.123, 1.7):
        ff_o = np.zeros(3 * g.n)
        out = oracle.alm(cs, st["u"], ff_o, t)
        ctx = make_ctx(case)
        ff_d = ctx.field(3)
        tq, th = ctx.alm_run(dev(ctx, st["u"]), ff_d, t)
        xyz, f, tqa, tha = ctx.alm_aps(case.alm.apcount)
        np.testing.assert_allclose(xyz, out["xyz"], rtol=1e-14, atol=1e-14)
        np.testing.assert_allclose(f, out["force"], rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(tq, out["torque"], rtol=1e-12)
        np.testing.assert_allclose(th, out["thrust"], rtol=1e-12)
        # projection truncated at 6 eps: relative L2 far below the FP64 budget
        assert rel_l2(interior(host(ff_d), g, 3), interior(ff_o, g, 3)) < 1e-13


def test_alm_pitch_motion(oracle, lib_built):
    """platform pitch motion (src/alm/almDevCall.cu:43-61, src/falmath.h:412-460)"""
    case = cases.small_channel(40, 28, 28, intensity=0.0)
    a = case.alm
    a.motion = np.array([[np.radians(3.0), 2 * np.pi / 10.0, 0.3]])
    a.angle_type = np.array([2], dtype=np.int32)
    a.hub = np.array([[0.0, 0.0, 0.5]])
    a.base = a.base - np.array([[0.0, 0.0, 0.5]])
    a.pitch = 2.0
    cs, m = _setup(oracle, case)
    st = random_state(case, seed=22, amp=0.05)
    ff_o = np.zeros(3 * case.grid.n)
    out = oracle.alm(cs, st["u"], ff_o, 2.5)
    ctx = make_ctx(case)
    tq, th = ctx.alm_run(dev(ctx, st["u"]), None, 2.5)
    np.testing.assert_allclose(tq, out["torque"], rtol=1e-12)
    np.testing.assert_allclose(th, out["thrust"], rtol=1e-12)


def test_mixed_solve_long_channel_stays_finite(lib_built):
    """The mixed-precision PBiCGStab on the nearly singular operator of a long
    channel (512x128x128, one Dirichlet face) with a smooth unit-norm
    right-hand side, which FP64 solves in about 240 iterations to a relative
    residual of 1e-2: FP32 recursions of that length diverge, so the solve
    replaces the recursive residual by the FP64 true one every 50 iterations.
    It must end with finite iterates and meet the relative residual 1e-2 within
    maxit 1000, and a relative residual of 1e-5, below what an FP32 iterate
    of this smooth solution can hold, must end at maxit (status 5) with finite
    iterates instead of non-finite scalars."""
    from falm_b200.api import _ptr
    case = cases.channel(512, 128, 128, cells_per_radius=20, tol=1e-6)
    g = case.grid
    ctx = make_ctx(case, "mixed")
    N = g.interior[0] * g.interior[1] * g.interior[2]
    z, y, x = np.meshgrid(np.arange(g.sz), np.arange(g.sy), np.arange(g.sx), indexing="ij")
    b = np.exp(-(((x - 64) / 6.0) ** 2 + ((y - g.sy / 2) / 6.0) ** 2 + ((z - g.sz / 2) / 6.0) ** 2))
    gc = g.gc
    b[:gc] = b[-gc:] = 0
    b[:, :gc] = b[:, -gc:] = 0
    b[:, :, :gc] = b[:, :, -gc:] = 0
    b /= np.linalg.norm(b)
    bt = dev(ctx, b.reshape(-1))
    for rel, want in ((1e-2, (0,)), (1e-5, (5,))):
        ctx.eq_init(1000, rel / N, case.pc, case.pc_maxit, case.pc_relax)
        xt, r = ctx.field(1), ctx.field(1)
        it, err = ctypes.c_int(), ctypes.c_double()
        rc = ctx.lib.falm_eq_solve(ctx.h, _ptr(xt), _ptr(bt), _ptr(r), ctx.stream(), ctypes.byref(it), ctypes.byref(err))
        assert rc in want, (rel, rc, it.value, err.value * N)
        assert np.isfinite(host(xt)).all() and np.isfinite(err.value)
        if rc == 0:
            assert err.value * N <= rel
    ctx.close()
