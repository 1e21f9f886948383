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


def test_mixed_precision_adjoint(lib_built):
    """The adjoint in a mixed-precision context -- FP32 forward steps, states
    and checkpoints; FP64 adjoint fields, gradient and transposed Poisson
    solve -- on the adjoint configuration (128x64x64, rotor of radius 10
    cells, seeded inflow), 20 steps from a spun-up state at the configuration's
    Poisson tolerance 1e-8.
      * The mixed adjoint along the mixed trajectory equals the FP64 context's
        adjoint evaluated at the same (FP32) states, step by step, to 1e-6
        relative (both transposed solves to relative residual 1e-9).
      * Against the FP64 run from the same start (a trajectory that differs by
        the mixed step's rounding and solver truncation): J within 1e-4, the
        gradient within 1e-2 relative.
      * Binomial checkpointing in the mixed context (3 stored states) gives the
        periodic checkpointing's objective to 1e-12 and its gradient to 1e-9."""
    import torch
    case = cases.adjoint_case().with_inflow()
    s64 = Simulation(case, "fp64")
    for _ in range(10):
        s64.step()
    start, it0 = A._clone(s64), s64.it
    s32 = Simulation(case, "mixed")

    def to_start(sim):
        for k in A.FIELDS:
            getattr(sim, k).copy_(start[k].to(sim.u.dtype))
        sim.it = it0

    steps, apc, n, dt = 20, case.alm.apcount, case.grid.n, case.dt
    # the mixed trajectory, every state kept
    to_start(s32)
    states = []
    for _ in range(steps):
        states.append(A._clone(s32))
        s32.step()
    states.append({"u": s32.u.clone()})

    def reverse(ctx, dtype):
        z = lambda m: torch.zeros(m, dtype=torch.float64, device=ctx.device)
        au, auu, anut, grad = z(3 * n), z(3 * n), z(n), z(1 + 2 * apc)
        for q in reversed(range(steps)):
            S = {k: v.to(dtype) for k, v in states[q].items()}
            ctx.step_adjoint(S["u"], S["uu"], S["p"], S["nut"], dt, (it0 + q + 1) * dt, 1.0 / steps, au, auu, anut, grad,
                             u_after=states[q + 1]["u"].to(dtype))
        return grad.cpu().numpy()

    s32.ctx.adjoint_set_tol(1e-9)
    s64.ctx.adjoint_set_tol(1e-9)
    g32 = reverse(s32.ctx, torch.float32)
    g64 = reverse(s64.ctx, torch.float64)
    assert g32[0] == pytest.approx(g64[0], rel=1e-6)
    for sl in (slice(1, 1 + apc), slice(1 + apc, None)):
        assert np.linalg.norm(g32[sl] - g64[sl]) <= 1e-6 * np.linalg.norm(g64[sl]), \
            np.linalg.norm(g32[sl] - g64[sl]) / np.linalg.norm(g64[sl])
    # the drivers: FP64 and mixed from the same start; binomial in mixed (the
    # transposed solves stay at 1e-9, so that their warm starts, which differ
    # between the runs, do not show)
    to_start(s64)
    J64, gp64, gc64, gt64 = A.mean_power_gradient(s64, steps, checkpoint=steps)
    to_start(s32)
    J32, gp32, gc32, gt32 = A.mean_power_gradient(s32, steps, checkpoint=5)
    assert J32 == pytest.approx(J64, rel=1e-4)
    assert gp32 == pytest.approx(gp64, rel=1e-2)
    for a, b in ((gc32, gc64), (gt32, gt64)):
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b), np.linalg.norm(a - b) / np.linalg.norm(b)
    to_start(s32)
    Jb, gpb, gcb, gtb = A.mean_power_gradient_binomial(s32, steps, snaps=3)
    assert Jb == pytest.approx(J32, rel=1e-12)
    assert gpb == pytest.approx(gp32, rel=1e-9)
    np.testing.assert_allclose(gcb, gc32, rtol=1e-9, atol=1e-12 * np.abs(gc32).max())
    np.testing.assert_allclose(gtb, gt32, rtol=1e-9, atol=1e-12 * np.abs(gt32).max())
    print("mixed vs fp64 trajectory: J", J32 / J64 - 1, "pitch", gp32 / gp64 - 1,
          "chord", np.linalg.norm(gc32 - gc64) / np.linalg.norm(gc64))
    s64.close()
    s32.close()
