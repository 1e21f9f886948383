"""The FP64 CPU discrete adjoint of the step (oracle_step_adjoint) against
central finite differences of the oracle's own step.

Objective: mean rotor power over a few steps from a spun-up state of a small
channel with the rotor and seeded inflow.  The Poisson solve runs to 1e-15 so
that it is exact to rounding, which is what the adjoint assumes.  The adjoint
gradients with respect to the collective pitch and per-actuator-point chord
and twist agree with central differences (step 1e-4) to 1e-6 relative; about
5% of each gradient comes through the flow (the rest is the direct blade
force term), so the flow adjoint is exercised."""
import numpy as np
import pytest

from falm_b200 import cases


@pytest.fixture(scope="module")
def setup(oracle):
    from oracle.oracle import CaseStruct
    case = cases.small_channel(24, 16, 16, cells_per_radius=5, intensity=0.05, n_ap_per_blade=6).with_inflow()
    cs = CaseStruct(case, maxit=400, tol=1e-15)
    m = oracle.setup(cs)
    st = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in cases.initial_state(case).items()}
    oracle.init_state(cs, m, st)
    for q in range(4):
        oracle.step(cs, st, m, (q + 1) * case.dt)
    return cs, m, st


def test_oracle_adjoint_matches_finite_differences(oracle, setup):
    cs, m, st = setup
    steps, it0, h = 4, 4, 1e-4
    J, gp, gch, gtw = oracle.adjoint(cs, m, st, steps, it0)
    assert J > 0

    def fd(bump):
        bump(+h)
        jp = oracle.objective(cs, m, st, steps, it0)
        bump(-2 * h)
        jm = oracle.objective(cs, m, st, steps, it0)
        bump(+h)
        return (jp - jm) / (2 * h)

    def pitch(d):
        cs.c.alm.pitch += d
    assert gp == pytest.approx(fd(pitch), rel=1e-6)
    ch, tw = cs.alm_arrays["ap_chord"], cs.alm_arrays["ap_twist"]
    for ap in (2, 7, 13):
        def chord(d, ap=ap):
            ch[ap] += d

        def twist(d, ap=ap):
            tw[ap] += d
        assert gch[ap] == pytest.approx(fd(chord), rel=1e-6)
        assert gtw[ap] == pytest.approx(fd(twist), rel=1e-6, abs=1e-10)
