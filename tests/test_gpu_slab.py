"""The step on a grid split into z slabs (falm_slab_init), on one GPU: the slabs
are contexts of this process, one host thread and CUDA stream each, joined by
the in-process transport (falm_local_hub); every exchange and reduction is a
host rendezvous plus event-ordered copies, and no kernel waits on another.

  * 2 and 3 slabs against 1 slab of the same slab path: the fields after 10
    FP64 steps in fixed-iteration mode (tol 0, maxit 6) within 1e-12 relative
    L2 (only the summation order of the reductions differs; the pressure, the
    BiCGStab iterate, within 1e-10: six Krylov iterations amplify the
    reductions' rounding to about 1e-11 there; the cavity see below), the same
    iteration counts, torque and thrust within 1e-12;
  * the slab path against the one-GPU step of falm_step (blocked red-black SOR,
    fused passes): within 1e-10 (rounding of the two preconditioner kernels);
  * the drivers' convergence mode: iteration counts within +-1;
  * mixed precision: 2 slabs against 1 slab within 1e-5;
  * the NCCL transport with one rank (libnccl loaded at run time, a one-rank
    communicator): the slab step equals the local transport's."""
import numpy as np
import pytest

from falm_b200 import cases
from falm_b200 import slab as SL
from tests.helpers import rel_l2
from tests.test_gpu_step import compare, run_gpu

pytestmark = pytest.mark.gpu


def slab_cases():
    ch = cases.small_channel(32, 20, 24, intensity=0.05).with_inflow(nb=8)     # rotor, seeded inflow
    cav = cases.cavity(16)
    cav.tol = 1e-10
    return {"channel": ch, "cavity": cav}


@pytest.mark.parametrize("name", ["channel", "cavity"])
def test_slabs_match_one_slab_fixed_iterations(lib_built, name):
    """Channel: after 10 steps the velocities within 1e-12 and the pressure
    within 1e-10.  Cavity: its all-Neumann (singular) Poisson problem from a
    flow at rest makes six fixed BiCGStab iterations amplify the reductions'
    rounding by about 1e6 between steps 2 and 5 (measured: 3e-16 after 2 steps,
    8e-10 in u and 1e-8 in p after 5), so it is held to 1e-13 after 2 steps and
    to 1e-8 (velocities) and 1e-6 (pressure, determined up to the singular
    operator's null space) after 10; the one-slab path equals the one-GPU step
    bit for bit there."""
    case = slab_cases()[name]
    checks = ((10, 1e-12, 1e-10),) if name == "channel" else ((2, 1e-13, 1e-13), (10, 1e-8, 1e-6))
    for steps, bu, bp in checks:
        one, s1 = SL.run_slabs(case, 1, steps, maxit=6, tol=0.0)
        for n in (2, 3):
            got, sn = SL.run_slabs(case, n, steps, maxit=6, tol=0.0)
            err = compare(case, got, one)
            for k in ("u", "uu", "nut"):
                assert err[k] < bu, (steps, n, k, err)
            assert err["p"] < bp, (steps, n, err)
            for r in range(n):
                for a, b in zip(sn[r], s1[0]):
                    assert a["it"] == b["it"]
                    assert a["divnorm"] == pytest.approx(b["divnorm"], rel=max(1e-10, bu))
                    for x, y in zip(a["torque"] + a["thrust"], b["torque"] + b["thrust"]):
                        assert x == pytest.approx(y, rel=1e-12)
    # the one-slab path against the one-GPU step
    ref, rs, ctx = run_gpu(case, 10, maxit=6, tol=0.0)
    ctx.close()
    err = compare(case, one, ref)
    for k, v in err.items():
        assert v < 1e-10, (k, v, err)


def test_slabs_converged_and_mixed(lib_built):
    case = slab_cases()["channel"]
    case.tol = 1e-8
    one, s1 = SL.run_slabs(case, 1, 6)
    two, s2 = SL.run_slabs(case, 2, 6)
    for a, b in zip(s2[0], s1[0]):
        assert abs(a["it"] - b["it"]) <= 1
    err = compare(case, two, one)
    assert err["u"] < 1e-9 and err["p"] < 1e-5, err
    one_m, _ = SL.run_slabs(case, 1, 6, precision="mixed")
    two_m, _ = SL.run_slabs(case, 2, 6, precision="mixed")
    err = compare(case, two_m, one_m)
    assert err["u"] < 1e-5, err
    assert compare(case, two_m, one)["u"] < 2e-4


def test_slabs_with_rmcp_match_one_slab_and_the_driver(lib_built):
    """The RMCP rotor (48^3 channel, rotor in the middle, so its blades cross the
    slab interfaces): each slab paints and forces its own cells and the turbine
    sums are reduced over the slabs.  2 slabs against 1 slab after 5 FP64 steps
    in fixed-iteration mode within 1e-12 (velocities) and 1e-10 (pressure),
    torque and thrust within 1e-12; the one-slab path against the Python
    driver's fused one-GPU step (driver.Simulation) within 1e-10."""
    from falm_b200.driver import Simulation
    from tests.test_gpu_rmcp import rmcp_case
    case = rmcp_case(10.0)
    one, s1 = SL.run_slabs(case, 1, 5, maxit=6, tol=0.0)
    two, s2 = SL.run_slabs(case, 2, 5, maxit=6, tol=0.0)
    err = compare(case, two, one)
    for k in ("u", "uu", "nut"):
        assert err[k] < 1e-12, (k, err)
    assert err["p"] < 1e-10, err
    for r in range(2):
        for a, b in zip(s2[r], s1[0]):
            assert a["it"] == b["it"]
            assert b["torque"][0] > 0
            for x, y in zip(a["torque"] + a["thrust"], b["torque"] + b["thrust"]):
                assert x == pytest.approx(y, rel=1e-12)
    case.maxit, case.tol = 6, 0.0
    sim = Simulation(case)
    st = [sim.step() for _ in range(5)]
    got = {k: getattr(sim, k).double().cpu().numpy() for k in ("u", "uu", "p", "nut")}
    sim.ctx.close()
    err = compare(case, got, one)
    for k, v in err.items():
        assert v < 1e-10, (k, v, err)
    for a, b in zip(st, s1[0]):
        assert a["torque"][0] == pytest.approx(b["torque"][0], rel=1e-10)


def test_nccl_transport_one_rank(lib_built):
    """libnccl through the library (a one-rank communicator: no exchange, the
    reductions an identity): the slab step is the local transport's, and the
    transport is destroyed cleanly."""
    import torch
    import torch.distributed as dist
    from falm_b200 import _lib as L
    case = slab_cases()["channel"]
    ref, _ = SL.run_slabs(case, 1, 3, maxit=6, tol=0.0)
    lib = L.load()
    import ctypes
    raw = (ctypes.c_ubyte * 128)()
    assert lib.falm_nccl_unique_id(ctypes.byref(raw)) == L.FALM_OK
    t = L.Transport()
    assert lib.falm_nccl_transport_create(ctypes.byref(raw), 0, 1, ctypes.byref(t)) == L.FALM_OK
    sim = SL.SlabSimulation(case, 0, 1, t, "fp64", "cuda:0", maxit=6, tol=0.0)
    for _ in range(3):
        sim.step()
    got = SL.gather(case, [sim.state()])
    sim.close()
    assert lib.falm_nccl_transport_destroy(ctypes.byref(t)) == L.FALM_OK
    err = compare(case, got, ref)
    for k, v in err.items():
        assert v == 0.0, (k, v)
