"""Shared helpers of the test-suite (not collected)."""
import numpy as np


def view(a, grid, ncol):
    return np.asarray(a).reshape(ncol, grid.sz, grid.sy, grid.sx)


def interior(a, grid, ncol=1):
    g = grid.gc
    return view(a, grid, ncol)[:, g:-g, g:-g, g:-g]


def faces(a, grid, ncol=3):
    """the face map (interior + the lower boundary face) of a face field"""
    g = grid.gc
    return view(a, grid, ncol)[:, g - 1:-g, g - 1:-g, g - 1:-g]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    return num / den if den > 0 else num


def random_state(case, seed=7, amp=0.1):
    """a smooth-ish random velocity/pressure state for single-operator tests"""
    rng = np.random.default_rng(seed)
    n = case.grid.n
    u = np.zeros(3 * n)
    u[:n] = 1.0
    u += amp * rng.standard_normal(3 * n)
    return {"u": u, "uu": amp * rng.standard_normal(3 * n), "p": rng.standard_normal(n),
            "nut": 1e-3 * np.abs(rng.standard_normal(n)), "ff": amp * rng.standard_normal(3 * n)}


def make_ctx(case, precision="fp64"):
    """a falm_b200 context configured for a case (as the drivers' init does)"""
    from falm_b200.api import Context
    ctx = Context(case.grid, precision)
    ctx.cfd_init(case.Re, case.adv, case.sgs, case.Cs)
    ctx.eq_init(case.maxit, case.tol, case.pc, case.pc_maxit, case.pc_relax)
    ctx.bc_init(case.bc, case.u_inlet)
    ctx.poisson_operator(case.bc)
    if case.inflow is not None:
        ctx.set_inflow(case.inflow, float(case.grid.hx[case.grid.gc]))
    if case.alm is not None:
        ctx.alm_init(case.alm)
    return ctx


def dev(ctx, a):
    import torch
    return torch.as_tensor(np.asarray(a), dtype=ctx.dtype, device=ctx.device).contiguous()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.detach().double().cpu().numpy()
