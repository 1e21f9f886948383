"""Discrete adjoint of the step on the GPU (falm_step_adjoint + the checkpointed
driver in falm_b200.adjoint).

Objective: mean rotor power over a few steps of a small channel with the
rotor and seeded inflow, from a spun-up state, FP64, Poisson tolerance near
rounding (the adjoint treats the solve as exact).  Checked against
  * the FP64 CPU adjoint of the same discretisation (oracle_step_adjoint):
    objective to 1e-10, gradients to 1e-7 relative;
  * central finite differences of the GPU forward step (step 1e-4):
    1e-5 relative;
  * itself with another checkpoint interval (recomputation is exact), and the
    torch.autograd wrapper's backward."""
import numpy as np
import pytest

from falm_b200 import adjoint as A
from falm_b200 import cases
from falm_b200.driver import Simulation

pytestmark = pytest.mark.gpu

STEPS = 4


def make_case():
    case = cases.small_channel(24, 16, 16, cells_per_radius=5, intensity=0.05, n_ap_per_blade=6).with_inflow()
    case.tol, case.maxit = 1e-15, 400
    return case


@pytest.fixture(scope="module")
def run(lib_built):
    case = make_case()
    sim = Simulation(case, "fp64")
    for _ in range(4):
        sim.step()
    start = (sim.it, A._clone(sim))
    J, gp, gc, gt = A.mean_power_gradient(sim, STEPS, checkpoint=2)
    return case, sim, start, J, gp, gc, gt


def restart(sim, start):
    A._restore(sim, start[1])
    sim.it = start[0]


def test_adjoint_matches_cpu_adjoint(oracle, run):
    from oracle.oracle import CaseStruct
    case, sim, start, J, gp, gc, gt = run
    cs = CaseStruct(case, maxit=400, tol=1e-15)
    m = oracle.setup(cs)
    st = {k: start[1][k].cpu().numpy().astype(np.float64).copy() for k in A.FIELDS}
    st["ff"] = np.zeros(3 * case.grid.n)
    Jo, gpo, gco, gto = oracle.adjoint(cs, m, st, STEPS, start[0])
    assert J == pytest.approx(Jo, rel=1e-10)
    assert gp == pytest.approx(gpo, rel=1e-7)
    np.testing.assert_allclose(gc, gco, rtol=1e-7, atol=1e-7 * np.abs(gco).max())
    np.testing.assert_allclose(gt, gto, rtol=1e-7, atol=1e-7 * np.abs(gto).max())


def test_adjoint_matches_finite_differences(run):
    case, sim, start, J, gp, gc, gt = run
    p0 = A.parameters(sim)
    apc = case.alm.apcount
    h = 1e-4

    def J_at(params):
        A._set_params(sim, params)
        restart(sim, start)
        return A.objective(sim, STEPS)

    for idx, adj in ((0, gp), (1 + 3, gc[3]), (1 + 11, gc[11]), (1 + apc + 5, gt[5]), (1 + apc + 14, gt[14])):
        pp, pm = p0.copy(), p0.copy()
        pp[idx] += h
        pm[idx] -= h
        fd = (J_at(pp) - J_at(pm)) / (2 * h)
        assert adj == pytest.approx(fd, rel=1e-5, abs=1e-9), idx
    A._set_params(sim, p0)


def test_checkpoint_interval_and_autograd_wrapper(run):
    import torch
    case, sim, start, J, gp, gc, gt = run
    restart(sim, start)
    J2, gp2, gc2, gt2 = A.mean_power_gradient(sim, STEPS, checkpoint=STEPS)
    assert J2 == pytest.approx(J, rel=1e-13)
    assert gp2 == pytest.approx(gp, rel=1e-9)
    np.testing.assert_allclose(gc2, gc, rtol=1e-9, atol=1e-12)
    MeanPower = A.make_mean_power(torch)
    params = torch.tensor(A.parameters(sim), dtype=torch.float64, requires_grad=True)
    Jt = MeanPower.apply(params, sim, start, STEPS, 2)
    Jt.backward()
    assert float(Jt.detach()) == pytest.approx(J, rel=1e-12)
    assert float(params.grad[0]) == pytest.approx(gp, rel=1e-9)


def test_step_adjoint_with_and_without_the_next_state(run):
    """falm_step_adjoint gives the same result whether it recomputes the step or is
    handed the velocity after it"""
    import torch
    case, sim, start, J, gp, gc, gt = run
    restart(sim, start)
    S = A._clone(sim)
    sim.step()
    u1 = sim.u.clone()
    n, apc, dt = case.grid.n, case.alm.apcount, case.dt
    out = []
    for ua in (None, u1):
        rng = np.random.default_rng(3)
        au = torch.tensor(rng.standard_normal(3 * n), dtype=torch.float64, device=sim.ctx.device)
        auu = torch.tensor(rng.standard_normal(3 * n), dtype=torch.float64, device=sim.ctx.device)
        anut = torch.tensor(rng.standard_normal(n), dtype=torch.float64, device=sim.ctx.device)
        grad = torch.zeros(1 + 2 * apc, dtype=torch.float64, device=sim.ctx.device)
        sim.ctx.step_adjoint(S["u"], S["uu"], S["p"], S["nut"], dt, (start[0] + 1) * dt, 1.0, au, auu, anut, grad, u_after=ua)
        out.append([x.cpu().numpy() for x in (au, auu, anut, grad)])
    for a, b in zip(*out):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9 * np.abs(b).max())


@pytest.mark.parametrize("snaps", [0, 1, 3])
def test_binomial_checkpointing_matches_keep_all(run, snaps):
    """Binomial checkpointing (at most `snaps` stored states besides the start,
    the end and one scratch state, steps recomputed along the optimal binomial
    schedule) gives the objective and gradient of the keep-everything reversal
    over a 9-step window: the forward steps are deterministic, so only the
    transposed solves' warm starts differ (within their tolerance)."""
    case, sim, start, J, gp, gc, gt = run
    restart(sim, start)
    Jk, gpk, gck, gtk = A.mean_power_gradient(sim, 9, checkpoint=9)
    end_u = sim.u.clone()
    restart(sim, start)
    Jb, gpb, gcb, gtb = A.mean_power_gradient_binomial(sim, 9, snaps=snaps)
    assert Jb == pytest.approx(Jk, rel=1e-14)
    assert gpb == pytest.approx(gpk, rel=1e-9)
    np.testing.assert_allclose(gcb, gck, rtol=1e-9, atol=1e-12 * np.abs(gck).max())
    np.testing.assert_allclose(gtb, gtk, rtol=1e-9, atol=1e-12 * np.abs(gtk).max())
    assert sim.it == start[0] + 9
    assert np.array_equal(sim.u.cpu().numpy(), end_u.cpu().numpy())


def test_adjoint_at_the_adjoint_configuration_size_matches_fd(lib_built):
    """The adjoint configuration at its own size and length: 128x64x64 channel,
    rotor of radius 10 cells with 3 x 32 actuator points, seeded 5% inflow,
    J = mean rotor power over 200 steps from a spun-up state, a checkpoint every
    20 steps with recomputation in between, the default transposed-solve
    tolerance (relative 1e-5).  The forward Poisson solve runs at err 1e-13 here
    so that J is a smooth function of the parameters (at 1e-8, iteration-count
    changes make central differences of J noisy at the 1e-4 level).
    Central differences (step 1e-4 for the collective pitch and the chord of
    two actuator points; 1e-3 for their twist, whose derivatives are 100x
    smaller, so that the difference of J stands above the solver's noise) agree
    with the adjoint gradient to 1e-4 relative."""
    case = cases.adjoint_case().with_inflow()
    case.tol, case.maxit = 1e-13, 2000
    sim = Simulation(case, "fp64")
    for _ in range(10):
        sim.step()
    start = (sim.it, A._clone(sim))
    steps, apc = 200, case.alm.apcount
    J, gp, gc, gt = A.mean_power_gradient(sim, steps, checkpoint=20)
    p0 = A.parameters(sim)

    def J_at(params):
        A._set_params(sim, params)
        restart(sim, start)
        return A.objective(sim, steps)

    for idx, adj, h in ((0, gp, 1e-4), (1 + 20, gc[20], 1e-4), (1 + 57, gc[57], 1e-4),
                        (1 + apc + 20, gt[20], 1e-3), (1 + apc + 57, gt[57], 1e-3)):
        pp, pm = p0.copy(), p0.copy()
        pp[idx] += h
        pm[idx] -= h
        fd = (J_at(pp) - J_at(pm)) / (2 * h)
        assert adj == pytest.approx(fd, rel=1e-4), (idx, adj, fd)
    A._set_params(sim, p0)
    sim.close()
