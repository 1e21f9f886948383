"""The RMCP rotor model (the reference's alternate forcing, src/rmcp/): the
rotating blades of each turbine paint the cells they cover and every painted
cell gets the blade-element force of its own velocity.

  * the paint and the force field of the B200 kernel, of the CPU oracle and of
    the reference's own RmcpAlm (oracle/_ref, SetALMFlag + ALM) on the same
    velocity field: identical paint, forces within 1e-13 relative L2; torque
    and thrust (B200 against the oracle) within 1e-12; an unyawed and a yawed
    turbine at two rotor angles;
  * the step with the RMCP forcing (FP64, fixed iterations) against the oracle's
    step fed with the oracle's RMCP force: 1e-10, torque within 1e-10; mixed
    precision within 2e-4 of it."""
import os

import numpy as np
import pytest

from falm_b200 import cases
from tests.helpers import dev, host, interior, make_ctx, random_state, rel_l2
from tests.test_gpu_step import compare

pytestmark = pytest.mark.gpu

REF_SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libfalmref.so")


def rmcp_case(yaw=0.0):
    """a 48^3 channel at 20 cells per rotor radius (the blade strip, 0.1 R wide and
    thick, covers two cells across), the rotor in the middle"""
    case = cases.small_channel(48, 48, 48, cells_per_radius=20, intensity=0.0)
    case.alm = None
    case.rmcp = cases.make_rmcp((1.2, 1.2, 1.2), yaw_deg=yaw)
    return case


@pytest.mark.parametrize("yaw", [0.0, 10.0])
@pytest.mark.parametrize("t", [0.0, 0.37])
def test_rmcp_force_matches_reference_and_oracle(oracle, lib_built, yaw, t):
    import tempfile
    import torch
    from oracle.oracle import CaseStruct, RefStep
    case = rmcp_case(yaw)
    g = case.grid
    st = random_state(case, seed=21, amp=0.05)
    cs = CaseStruct(case)
    ff_o, flag_o, tq_o, th_o = oracle.rmcp(cs, case.rmcp, st["u"], t)
    fo = interior(flag_o, g)
    assert 50 < np.count_nonzero(fo) < fo.size // 10     # some cells painted, the rest not
    ctx = make_ctx(case)
    ctx.rmcp_init(case.rmcp)
    ff = ctx.field(3)
    flag = torch.zeros(g.n, dtype=torch.int32, device=ctx.device)
    tq, th = ctx.rmcp_run(dev(ctx, st["u"]), ff, t, flag)
    np.testing.assert_array_equal(interior(flag.cpu().numpy(), g), fo)
    assert rel_l2(interior(host(ff), g, 3), interior(ff_o, g, 3)) < 1e-13
    assert tq[0] == pytest.approx(tq_o[0], rel=1e-12) and th[0] == pytest.approx(th_o[0], rel=1e-12)
    ctx.close()
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref not built")
    ref = RefStep(CaseStruct(case, use_inflow=False), tempfile.mkdtemp(prefix="falmref_"))
    ref.rmcp_init(case.rmcp)
    ref.set("U", st["u"])
    ff_r, flag_r = ref.rmcp_run(t)
    ref.close()
    np.testing.assert_array_equal(interior(flag_r, g), fo)
    assert rel_l2(interior(ff_o, g, 3), interior(ff_r, g, 3)) < 1e-13


def run_rmcp_oracle(oracle, case, steps, fixed=True):
    from oracle.oracle import CaseStruct
    cs = CaseStruct(case, maxit=6, tol=0.0) if fixed else CaseStruct(case)
    m = oracle.setup(cs)
    st = cases.initial_state(case)
    oracle.init_state(cs, m, st)
    torques = []
    for q in range(steps):
        t = (q + 1) * case.dt
        ff, _, tq, _ = oracle.rmcp(cs, case.rmcp, st["u"], t)
        st["ff"] = ff
        oracle.step(cs, st, m, t)
        torques.append(tq[0])
    return st, torques


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rmcp_step_matches_oracle(oracle, lib_built, precision):
    """FP64 in fixed-iteration mode (tol 0, maxit 6); mixed precision in the
    drivers' convergence mode (tol 1e-8; its FP64 refinement needs a tolerance)"""
    case = rmcp_case(10.0)
    fixed = precision == "fp64"
    case.tol = 1e-8
    ref, tq_ref = run_rmcp_oracle(oracle, case, 5, fixed)
    ctx = make_ctx(case, precision)
    if fixed:
        ctx.eq_init(6, 0.0, case.pc, case.pc_maxit, case.pc_relax)
    ctx.rmcp_init(case.rmcp)
    st0 = cases.initial_state(case)
    u, uu, p, nut = dev(ctx, st0["u"]), ctx.field(3), ctx.field(1), ctx.field(1)
    ctx.utouu(u, uu)
    ctx.sgs(u, nut)
    stats = [ctx.step(u, uu, p, nut, None, case.dt, (q + 1) * case.dt) for q in range(5)]
    got = {"u": host(u), "uu": host(uu), "p": host(p), "nut": host(nut)}
    ctx.close()
    err = compare(case, got, ref)
    if precision == "fp64":
        for k, v in err.items():
            assert v < 1e-10, (k, v, err)
        for s, tq in zip(stats, tq_ref):
            assert s["torque"][0] == pytest.approx(tq, rel=1e-10)
    else:
        assert err["u"] < 2e-4 and err["uu"] < 2e-4, err
        for s, tq in zip(stats, tq_ref):
            assert s["torque"][0] == pytest.approx(tq, rel=5e-3)
