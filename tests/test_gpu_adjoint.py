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
