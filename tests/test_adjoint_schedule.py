"""Binomial checkpointing of the adjoint driver (falm_b200.adjoint), on the CPU.

A stand-in simulation with a deterministic step (torch CPU tensors) and a
stand-in context that records every falm_step_adjoint call check the schedule
itself: for every window length and number of slots, each step is reversed
exactly once, last step first, with the state before it and the velocity after
it equal to those of a plain forward run; the objective equals the plain run's
mean power; the simulation ends after the window; the number of forward steps
equals the dynamic programme's count, which never exceeds the schedule that
restarts from the window's start for every step and, with enough slots,
reaches the keep-everything minimum (one forward step per step plus one
advance per stored state)."""
import types

import numpy as np
import pytest

from falm_b200 import adjoint as A


class FakeCtx:
    def __init__(self, torch):
        self.torch = torch
        self.precision = "fp64"
        self.device = "cpu"
        self.calls = []

    def step_adjoint(self, u, uu, p, nut, dt, t, w_power, au, auu, anut, grad, u_after=None):
        self.calls.append((round(t / dt), u.clone(), u_after.clone()))
        grad[0] += w_power


class FakeSim:
    def __init__(self, torch, n=5):
        self.torch = torch
        self.ctx = FakeCtx(torch)
        self.case = types.SimpleNamespace(dt=0.5, grid=types.SimpleNamespace(n=n),
                                          alm=types.SimpleNamespace(tip_rate=[2.0], apcount=1))
        self.u = torch.arange(3 * n, dtype=torch.float64) * 0.1
        self.uu = torch.zeros(3 * n, dtype=torch.float64)
        self.p = torch.zeros(n, dtype=torch.float64)
        self.nut = torch.zeros(n, dtype=torch.float64)
        self.it = 3
        self.forward_steps = 0

    def step(self):
        self.it += 1
        self.forward_steps += 1
        self.u.mul_(1.01).add_(0.001 * self.it)
        self.uu.copy_(self.u * 0.5)
        self.p.add_(self.u[: self.p.numel()])
        self.nut.copy_(self.p.abs() * 1e-3)
        return {"torque": [float(self.u.sum())], "thrust": [0.0]}


@pytest.mark.parametrize("steps", [1, 2, 7, 20, 33])
@pytest.mark.parametrize("snaps", [0, 1, 2, 5, 40])
def test_binomial_reversal_order_states_and_cost(steps, snaps):
    torch = pytest.importorskip("torch")
    ref = FakeSim(torch)
    states, power = [], []
    for _ in range(steps):
        states.append(ref.u.clone())
        power.append(2.0 * ref.step()["torque"][0])
    states.append(ref.u.clone())
    sim = FakeSim(torch)
    J, gp, gc, gt = A.mean_power_gradient_binomial(sim, steps, snaps=snaps)
    assert J == pytest.approx(float(np.mean(power)), rel=1e-15)
    calls = sim.ctx.calls
    assert [c[0] for c in calls] == [3 + a + 1 for a in reversed(range(steps))]
    for (t, u0, u1), a in zip(calls, reversed(range(steps))):
        assert torch.equal(u0, states[a]) and torch.equal(u1, states[a + 1])
    assert sim.it == 3 + steps and torch.equal(sim.u, states[-1])
    assert gp == pytest.approx(1.0)
    s = max(0, min(snaps, steps - 1))
    assert sim.forward_steps == A.binomial_forward_steps(steps, s)
    assert sim.forward_steps <= steps + steps * (steps - 1) // 2
    if s >= steps - 1:
        assert sim.forward_steps == 2 * steps - 1


def test_binomial_table_properties():
    """The dynamic programme's advance counts: t (t - 1) / 2 with no free slot,
    t - 1 (every state stored once) with t - 1 slots or more, never more with
    more slots, and the hand-counted schedules of small windows (3 steps, one
    slot: 2; 4 steps, one slot: 4; 4 steps, two slots: 3)."""
    G, split = A.binomial_table(60, 12)
    for t in range(1, 61):
        assert G[t, 0] == t * (t - 1) // 2
        for s in range(1, 13):
            assert G[t, s] <= G[t, s - 1]
            if s >= t - 1:
                assert G[t, s] == max(t - 1, 0)
            if t >= 2:
                assert 1 <= split[t, s] < t
    assert (G[3, 1], G[4, 1], G[4, 2]) == (2, 4, 3)
