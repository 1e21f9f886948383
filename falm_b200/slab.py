"""Z-slab decomposition of the LES step over several GPUs.

The reference splits its grid into per-rank boxes with an MPI halo exchange
(CPM: src/CPMBase.h:36-112, src/CPMComm.h:182-364; its drivers split x,
app/nedo/main.cpp:105).  Here the grid is split along z into slabs of whole
planes, one per GPU: every halo is a run of contiguous planes of each
component, and the library's step exchanges them and reduces every inner
product, norm and actuator-point force over the slabs through a transport
(falm_slab_init, include/falm_b200.h).

  partition(nz, nranks)           the slabs' (z_offset, nz_local), balanced
  slab_grid(grid, z0, nzl)        the grid of one slab (guide planes included)
  slab_case(case, z0, nzl)        the case on that grid (same rotor and inflow)
  LocalHub(nranks)                the in-process transport (one thread per rank)
  nccl_transport(rank, nranks)    the NCCL transport (one process per GPU, after
                                  torch.distributed.init_process_group)
  SlabSimulation                  one rank's slab: context, fields and step
  run_slabs(case, nranks, steps)  nranks slabs as threads of this process,
                                  gathered into whole-grid fields
"""
import ctypes
import dataclasses
import threading

import numpy as np

from . import _lib as L
from . import cases as C
from .api import Context


def partition(nz, nranks):
    """(z_offset, nz_local) of each rank: nz interior planes split as evenly as
    possible, the larger slabs first; every slab holds at least two planes (the
    depth of the velocity's halo)"""
    if nranks < 1 or nz < 2 * nranks:
        raise ValueError(f"cannot split {nz} planes into {nranks} slabs of at least 2")
    base, extra = divmod(nz, nranks)
    out, z0 = [], 0
    for r in range(nranks):
        n = base + (1 if r < extra else 0)
        out.append((z0, n))
        z0 += n
    return out


def slab_grid(grid, z0, nzl):
    """the slab of interior planes [z0, z0 + nzl) with its guide planes: across a
    slab interface the guide planes are the neighbour's interior planes, so the
    coordinate and width arrays are the whole grid's there"""
    gc = grid.gc
    sl = slice(z0, z0 + nzl + 2 * gc)
    return C.Grid(grid.sx, grid.sy, nzl + 2 * gc, gc, grid.x, grid.y, grid.z[sl].copy(), grid.hx, grid.hy, grid.hz[sl].copy())


def slab_case(case, z0, nzl):
    """the case on one slab; its inflow box and rotor are the whole grid's"""
    return dataclasses.replace(case, grid=slab_grid(case.grid, z0, nzl))


class LocalHub:
    """falm_local_hub: the transport between the slabs of one process"""

    def __init__(self, nranks):
        self.lib = L.load()
        h = ctypes.c_void_p()
        rc = self.lib.falm_local_hub_create(nranks, ctypes.byref(h))
        if rc:
            raise L.FalmError(rc, "falm_local_hub_create")
        self.h, self.nranks = h, nranks

    def transport(self, rank):
        t = L.Transport()
        rc = self.lib.falm_local_hub_transport(self.h, rank, ctypes.byref(t))
        if rc:
            raise L.FalmError(rc, "falm_local_hub_transport")
        return t

    def close(self):
        if self.h:
            self.lib.falm_local_hub_destroy(self.h)
            self.h = None


def broadcast_id(id_bytes, src=0):
    """the 128 bytes of rank `src` on every rank of the default torch.distributed
    group (a uint8 tensor on the group's device)"""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.zeros(128, dtype=torch.uint8, device=dev)
    if dist.get_rank() == src:
        t.copy_(torch.tensor(list(id_bytes), dtype=torch.uint8))
    dist.broadcast(t, src)
    return bytes(t.cpu().tolist())


def nccl_transport(rank, nranks):
    """falm_nccl_transport_create on every rank of an initialised torch.distributed
    group (one process per GPU, the current device set): rank 0's NCCL unique id
    is broadcast through the group (one rank needs no group)"""
    lib = L.load()
    raw = (ctypes.c_ubyte * 128)()
    if rank == 0:
        rc = lib.falm_nccl_unique_id(ctypes.byref(raw))
        if rc:
            raise L.FalmError(rc, "falm_nccl_unique_id")
    if nranks > 1:
        uid = broadcast_id(bytes(raw), 0)
        raw = (ctypes.c_ubyte * 128)(*uid)
    t = L.Transport()
    rc = lib.falm_nccl_transport_create(ctypes.byref(raw), rank, nranks, ctypes.byref(t))
    if rc:
        raise L.FalmError(rc, "falm_nccl_transport_create")
    return t


class SlabSimulation:
    """One rank's slab of a case: the init of app/nedo/main.cpp:102-133 on the
    slab (the operator build is a collective), then falm_step per step."""

    def __init__(self, case, rank, nranks, transport, precision="fp64", device=None, maxit=None, tol=None, perturb=None):
        nz = case.grid.interior[2]
        z0, nzl = partition(nz, nranks)[rank]
        self.case, self.rank, self.nranks, self.z0, self.nzl = case, rank, nranks, z0, nzl
        self.local = slab_case(case, z0, nzl)
        g = self.local.grid
        ctx = Context(g, precision, device)
        ctx.slab_init(rank, nranks, z0, nz, transport)
        ctx.cfd_init(case.Re, case.adv, case.sgs, case.Cs)
        ctx.eq_init(case.maxit if maxit is None else maxit, case.tol if tol is None else tol, case.pc, case.pc_maxit,
                    case.pc_relax)
        ctx.bc_init(case.bc, case.u_inlet)
        self.maxdiag = ctx.poisson_operator(case.bc)
        if case.inflow is not None:
            ctx.set_inflow(case.inflow, float(case.grid.hx[case.grid.gc]))
        if case.alm is not None:
            ctx.alm_init(case.alm)
        if getattr(case, "rmcp", None) is not None:
            ctx.rmcp_init(case.rmcp)
        self.ctx = ctx
        torch = ctx.torch
        st = C.initial_state(self.local)
        if perturb is not None:
            # u + eps N(0, 1) cell by cell (velocities are of order one), the noise drawn on the whole grid
            eps, seed = perturb
            gg = case.grid
            noise = np.random.default_rng(seed).standard_normal((3, gg.sz, gg.sy, gg.sx))[:, z0:z0 + g.sz]
            st["u"] = st["u"] + eps * noise.reshape(-1)
        self.u = torch.as_tensor(st["u"], dtype=ctx.dtype, device=ctx.device).contiguous()
        self.uu, self.p, self.nut = ctx.field(3), ctx.field(1), ctx.field(1)
        ctx.slab_halo(self.u, 2)
        ctx.utouu(self.u, self.uu)
        ctx.sgs(self.u, self.nut)
        self.it = 0

    def step(self):
        self.it += 1
        return self.ctx.step(self.u, self.uu, self.p, self.nut, None, self.case.dt, self.it * self.case.dt)

    def state(self):
        """host copies of the slab's fields (guide planes included)"""
        import torch
        torch.cuda.synchronize()
        return {k: getattr(self, k).double().cpu().numpy() for k in ("u", "uu", "p", "nut")}

    def close(self):
        self.ctx.close()


def gather(case, states):
    """whole-grid fields from the slabs' states: each slab's interior planes, and
    the guide planes of the lowest and highest slabs"""
    g = case.grid
    gc = g.gc
    nranks = len(states)
    parts = partition(g.interior[2], nranks)
    out = {}
    for k, nc in (("u", 3), ("uu", 3), ("p", 1), ("nut", 1)):
        a = np.zeros((nc, g.sz, g.sy, g.sx))
        for r, ((z0, nzl), st) in enumerate(zip(parts, states)):
            v = st[k].reshape(nc, nzl + 2 * gc, g.sy, g.sx)
            lo = 0 if r == 0 else gc
            hi = nzl + 2 * gc if r == nranks - 1 else nzl + gc
            a[:, z0 + lo:z0 + hi] = v[:, lo:hi]
        out[k] = a.reshape(-1)
    return out


def run_slabs(case, nranks, steps, precision="fp64", maxit=None, tol=None, device=None, perturb=None):
    """`steps` steps of the case split into nranks slabs, each driven by a thread
    of this process on its own CUDA stream of `device`; returns the gathered
    whole-grid fields and each rank's per-step statistics.  perturb = (eps,
    seed) adds eps N(0, 1) to the initial velocity cell by cell."""
    import torch
    dev = torch.device(device or "cuda:0")
    hub = LocalHub(nranks)
    results, errors = [None] * nranks, [None] * nranks

    def work(rank):
        try:
            torch.cuda.set_device(dev)
            stream = torch.cuda.Stream(dev)
            with torch.cuda.stream(stream):
                sim = SlabSimulation(case, rank, nranks, hub.transport(rank), precision, dev, maxit, tol, perturb)
                stats = [sim.step() for _ in range(steps)]
                results[rank] = (sim.state(), stats)
                sim.close()
        except Exception as e:   # reported on the calling thread
            errors[rank] = e

    threads = [threading.Thread(target=work, args=(r,)) for r in range(nranks)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    hub.close()
    for e in errors:
        if e is not None:
            raise e
    return gather(case, [r[0] for r in results]), [r[1] for r in results]
