"""Pin the CPU oracle against the known-answer material of the reference's own
test directory (test/dot.py, test/heat1d2.cpp, test/coloridx.py) and against
closed-form properties of the discretisation.  CPU only."""
import ctypes

import numpy as np
import pytest

from falm_b200 import cases
from tests.helpers import interior, rel_l2


def _box_case(shape, gc, h=1.0):
    """a case whose grid is an arbitrary box with `gc` guide cells"""
    def axis(n):
        return np.arange(n, dtype=np.float64) * h, np.full(n, h)
    x, hx = axis(shape[0])
    y, hy = axis(shape[1])
    z, hz = axis(shape[2])
    g = cases.Grid(shape[0], shape[1], shape[2], gc, x, y, z, hx, hy, hz)
    return cases.Case("box", g, 1, Re=100.0, dt=1e-3, tol=1e-9)


def test_dot_norm_quadratic_fields(oracle):
    """test/dot.py:15-30 and test/dot.cpp:9-37: interior-only dot product and
    squared norm of two quadratic fields on a 12^3 array with a 10^3 map."""
    from oracle.oracle import CaseStruct
    case = _box_case((12, 12, 12), 1)
    cs = CaseStruct(case)
    k, j, i = np.meshgrid(np.arange(12), np.arange(12), np.arange(12), indexing="ij")
    a = (300 - (i - 7) ** 2 - (j - 2) ** 2 - (k - 5) ** 2).astype(np.float64).ravel()
    b = (150 - (i - 0) ** 2 - (j - 1) ** 2 - (k - 1) ** 2).astype(np.float64).ravel()
    inside = ((i > 0) & (i < 11) & (j > 0) & (j < 11) & (k > 0) & (k < 11)).ravel()
    expect_ab = int(np.sum((a * b)[inside]))
    expect_aa = int(np.sum((a * a)[inside]))
    got_ab = oracle.L.oracle_dot(ctypes.byref(cs.c), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    got_aa = oracle.L.oracle_normsq(ctypes.byref(cs.c), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1)
    assert got_ab == expect_ab
    assert got_aa == expect_aa


def heat1d_system(nx=100, lx=1.0, tw=0.0, te=100.0, gd=2):
    """test/heat1d2.cpp:80-113 restated in the current column order (c,w,e,s,n,b,t):
    1D Dirichlet conduction with ghost reflection, then maxdiag scaling."""
    shape = (nx + 2 * gd, 1 + 2 * gd, 1 + 2 * gd)
    n = shape[0] * shape[1] * shape[2]
    A = np.zeros(7 * n)
    b = np.zeros(n)
    dx = lx / nx
    for i in range(gd, gd + nx):
        if i == gd:
            ae, aw, ac, bc = 1 / dx ** 2, 0.0, -(1 / dx ** 2 + 2 / dx ** 2), -(2 * tw) / dx ** 2
        elif i == gd + nx - 1:
            ae, aw, ac, bc = 0.0, 1 / dx ** 2, -(1 / dx ** 2 + 2 / dx ** 2), -(2 * te) / dx ** 2
        else:
            ae, aw, ac, bc = 1 / dx ** 2, 1 / dx ** 2, -(2 / dx ** 2), 0.0
        idx = i + gd * shape[0] + gd * shape[0] * shape[1]
        A[idx], A[idx + n], A[idx + 2 * n] = ac, aw, ae
        b[idx] = bc
    maxdiag = np.abs(A[:n]).max()
    A /= maxdiag
    b /= maxdiag
    exact = np.zeros(n)
    xs = (np.arange(nx) + 0.5) * dx
    for q, i in enumerate(range(gd, gd + nx)):
        exact[i + gd * shape[0] + gd * shape[0] * shape[1]] = tw + (te - tw) * xs[q] / lx
    return shape, A, b, exact


def test_heat1d_linear_profile(oracle):
    """test/heat1d2.cpp:217: PBiCGStab (maxit 1000, tol 1e-9) with SOR preconditioning
    (5 sweeps, omega 1.5) reproduces the linear Dirichlet profile."""
    from oracle.oracle import CaseStruct
    shape, A, b, exact = heat1d_system()
    case = _box_case(shape, 2, h=0.01)
    case.maxit, case.tol, case.pc, case.pc_maxit, case.pc_relax = 1000, 1e-9, "SOR", 5, 1.5
    cs = CaseStruct(case)
    x = np.zeros_like(b)
    r = np.zeros_like(b)
    it, err = oracle.pbicgstab(cs, A, x, b, r)
    assert err <= 1e-9 and it < 1000
    assert rel_l2(x, exact) < 1e-7


@pytest.mark.parametrize("ls,relax", [("Jacobi", 1.0), ("SOR", 1.8)])
def test_heat1d_plain_solvers(oracle, ls, relax):
    """FalmEq::Jacobi / FalmEq::SOR (src/FalmEq.cpp:80-127, :173-240) on the
    test/heat1d2.cpp system (20 cells) reproduce the linear Dirichlet profile,
    and the loop stops at the first iterate with ||r||/N <= tol."""
    from oracle.oracle import CaseStruct
    shape, A, b, exact = heat1d_system(nx=20)
    case = _box_case(shape, 2, h=0.05)
    case.maxit, case.tol = 100000, 1e-10
    x, r = np.zeros_like(b), np.zeros_like(b)
    it, err = oracle.plain_solve(CaseStruct(case), ls, relax, A, x, b, r)
    assert err <= 1e-10 and it < case.maxit
    assert rel_l2(x, exact) < 1e-6
    case.maxit = it - 1
    x2 = np.zeros_like(b)
    it2, err2 = oracle.plain_solve(CaseStruct(case), ls, relax, A, x2, b, r)
    assert it2 == it - 1 and err2 > 1e-10


def test_red_black_colouring(oracle):
    """src/dev/FalmEqDevCall.cu:206 and test/coloridx.py: colour (i+j+k+offset)%2,
    the black (0) half-sweep touches only colour-0 cells and leaves the others."""
    from oracle.oracle import CaseStruct, _p
    case = cases.cavity(8)
    cs = CaseStruct(case)
    m = oracle.setup(cs)
    rng = np.random.default_rng(1)
    g = case.grid
    x0 = rng.standard_normal(g.n)
    b = rng.standard_normal(g.n)
    for color in (0, 1):
        x = x0.copy()
        oracle.L.oracle_sor_sweep(ctypes.byref(cs.c), _p(m["A"]), _p(x), _p(b), 1.2, color)
        k, j, i = np.meshgrid(np.arange(g.sz), np.arange(g.sy), np.arange(g.sx), indexing="ij")
        inside = ((i >= 2) & (i < g.sx - 2) & (j >= 2) & (j < g.sy - 2) & (k >= 2) & (k < g.sz - 2)).ravel()
        on = (((i + j + k) % 2) == color).ravel() & inside
        changed = x != x0
        assert not changed[~on].any()
        assert changed[on].mean() > 0.99


def test_poisson_operator_rows(oracle):
    """app/nedo/main.cpp:25-100: uniform grid, interior rows are the scaled 7-point
    Laplacian; Neumann faces drop a coefficient except the x+ outlet (kept)."""
    from oracle.oracle import CaseStruct
    case = cases.small_channel(12, 8, 8, intensity=0.0)
    case.alm = None
    cs = CaseStruct(case)
    m = oracle.setup(cs)
    g = case.grid
    n = g.n
    A = m["A"].reshape(7, g.sz, g.sy, g.sx)
    h = g.hx[0]
    assert m["maxdiag"] == pytest.approx(6 / h ** 2, rel=1e-12)
    ci = A[:, 4, 4, 4]
    assert ci[0] == pytest.approx(-1.0, abs=1e-14) and np.allclose(ci[1:], 1 / 6, atol=1e-14)
    # x- face: west dropped; x+ face: east kept
    assert A[1, 4, 4, 2] == 0 and A[2, 4, 4, g.sx - 3] == pytest.approx(1 / 6)
    # y/z Neumann faces
    assert A[3, 4, 2, 4] == 0 and A[4, 4, g.sy - 3, 4] == 0 and A[5, 2, 4, 4] == 0 and A[6, g.sz - 3, 4, 4] == 0
    # row sums vanish on interior rows away from x+
    rs = A.sum(axis=0)[2:-2, 2:-2, 2:-3]
    assert np.abs(rs).max() < 1e-14


def test_projection_makes_faces_divergence_free(oracle):
    """With a tight Poisson solve the projected face velocities are discretely
    divergence free (the property the step's div norm reports)."""
    from oracle.oracle import CaseStruct, _p
    case = cases.small_channel(16, 10, 10, intensity=0.0)
    case.alm = None
    case.tol = 1e-13
    cs = CaseStruct(case)
    m = oracle.setup(cs)
    g = case.grid
    rng = np.random.default_rng(3)
    uu = rng.standard_normal(3 * g.n)
    rhs, res, div = np.zeros(g.n), np.zeros(g.n), np.zeros(g.n)
    p = np.zeros(g.n)
    c = ctypes.byref(cs.c)
    oracle.L.oracle_poisson_rhs(c, _p(uu), _p(rhs), _p(m["ja"]), m["maxdiag"])
    it, err = oracle.pbicgstab(cs, m["A"], p, rhs, res)
    oracle.L.oracle_pbc(c, _p(p))
    u = np.zeros(3 * g.n)
    oracle.L.oracle_project_p(c, _p(u), _p(u.copy()), _p(uu), _p(uu.copy()), _p(p), _p(m["kx"]), _p(m["g"]))
    oracle.L.oracle_divergence(c, _p(uu), _p(div), _p(m["ja"]))
    d0 = np.zeros(g.n)
    assert np.abs(interior(div, g)).max() < 1e-8


def test_build_aps_matches_python_restatement(oracle):
    """src/alm/bladeHandler.h:46-104 via the oracle and via the numpy restatement."""
    from oracle.oracle import _p
    st = cases.blade_stations()
    apc, nb = 96, 32
    ref = cases.build_aps_py(st, apc, nb, 1.0, 0.0)
    na = len(st["attack"])
    outs = [np.zeros(apc), np.zeros(apc), np.zeros(apc), np.zeros(apc * na), np.zeros(apc * na)]
    keep = [np.ascontiguousarray(st[k], dtype=np.float64) for k in ("r", "chord", "twist", "cl", "cd")]
    oracle.L.oracle_build_aps(2, *[_p(a) for a in keep], na, apc, nb, 1.0, 0.0, *[_p(a) for a in outs])
    for k, o in zip(("r", "chord", "twist", "cl", "cd"), outs):
        np.testing.assert_array_equal(o, ref[k])
    # hub radius 0: the first APs sit inside r/R < 0.1 and take the root station
    assert ref["chord"][0] == st["chord"][0] and ref["twist"][1] == st["twist"][0]


def test_alm_single_point_force(oracle):
    """src/alm/almDevCall.cu:131-253 on a uniform stream: every AP sees u = (1,0,0),
    phi = atan(1/(tip r)), lift/drag from the tabulated polar, projection integrates
    to the sum of AP forces."""
    from oracle.oracle import CaseStruct
    case = cases.small_channel(48, 32, 32, intensity=0.0)
    cs = CaseStruct(case)
    m = oracle.setup(cs)
    st = cases.initial_state(case)
    out = oracle.alm(cs, st["u"], st["ff"], 0.0)
    a = case.alm
    r = a.aps["r"]
    phi = np.arctan(1.0 / (7.0 * r))
    att = np.degrees(phi) - a.aps["twist"]
    cl = np.interp(att, a.stations["attack"], a.stations["cl"][0])
    cd = np.interp(att, a.stations["attack"], a.stations["cd"][0])
    urel2 = 1.0 + (7.0 * r) ** 2
    dr = 1.0 / a.n_ap_per_blade
    fl, fd = 0.5 * cl * urel2 * a.aps["chord"] * dr, 0.5 * cd * urel2 * a.aps["chord"] * dr
    fx = fl * np.cos(phi) + fd * np.sin(phi)
    ft = fl * np.sin(phi) - fd * np.sin(phi)
    np.testing.assert_allclose(out["thrust_ap"], fx, rtol=1e-12)
    np.testing.assert_allclose(out["torque_ap"], np.abs(ft) * r, rtol=1e-12)
    h = case.grid.hx[0]
    total = interior(st["ff"], case.grid, 3).reshape(3, -1).sum(axis=1) * h ** 3
    np.testing.assert_allclose(total, out["force"].sum(axis=0), rtol=2e-3, atol=1e-6)
