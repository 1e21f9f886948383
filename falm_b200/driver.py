"""Step driver: the init and time loop of app/nedo/main.cpp:102-236 (and
app/lid3d/main.cpp for the cavity) over the falm_b200 C ABI."""
import numpy as np

from . import cases as C
from .api import Context


class Simulation:
    def __init__(self, case, precision="fp64", fuse_alm=True, device=None):
        self.case = case
        ctx = Context(case.grid, precision, device)
        ctx.cfd_init(case.Re, case.adv, case.sgs, case.Cs)
        ctx.eq_init(case.maxit, case.tol, case.pc, case.pc_maxit, case.pc_relax)
        ctx.bc_init(case.bc, case.u_inlet)
        self.maxdiag = ctx.poisson_operator(case.bc)
        if case.inflow is not None:
            ctx.set_inflow(case.inflow, float(case.grid.hx[case.grid.gc]))
        if case.alm is not None:
            ctx.alm_init(case.alm)
        if getattr(case, "rmcp", None) is not None:
            ctx.rmcp_init(case.rmcp)        # the RMCP model replaces the ALM as the step's forcing
        self.ctx = ctx
        torch = ctx.torch
        st = C.initial_state(case)
        self.u = torch.as_tensor(st["u"], dtype=ctx.dtype, device=ctx.device).contiguous()
        self.uu, self.p, self.nut = ctx.field(3), ctx.field(1), ctx.field(1)
        rmcp = getattr(case, "rmcp", None) is not None
        self.ff = None if rmcp or (fuse_alm and case.alm is not None) else ctx.field(3)
        ctx.utouu(self.u, self.uu)         # app/nedo/main.cpp:132-133
        ctx.sgs(self.u, self.nut)
        self.it = 0

    def t(self):
        return self.it * self.case.dt

    def save_state(self, path):
        """a restart file of the step state (u, uu, p, nut: the snapshot format of
        FalmIO::writeVectorFile with the step index and time in its header),
        written before this returns"""
        self.ctx.write_vector_file(path, [self.u, self.uu, self.p, self.nut], self.it, self.t())
        self.ctx.io_wait()

    def load_state(self, path):
        """resume from a restart file of save_state (the same case and grid): the
        following steps continue the saved run exactly"""
        step, _ = self.ctx.read_vector_file(path, [self.u, self.uu, self.p, self.nut])
        self.it = int(step)

    def step(self):
        """one main_loop iteration (then TAvg and outputUVWP, app/nedo/main.cpp:199-200,
        when output is enabled); returns the step statistics"""
        self.it += 1
        st = self.ctx.step(self.u, self.uu, self.p, self.nut, self.ff, self.case.dt, self.t())
        out = getattr(self, "_out", None)
        if out is not None:
            self._output_step(out)
        return st

    def enable_output(self, prefix, interval, start=0, end=None, tavg_start=None, tavg_end=None, as_fp64=False):
        """FalmSolver's output schedule (src/falm.h:83-98, 433-475): after step it,
        TAvg of u and p while tavg_start <= it <= tavg_end, and when
        start <= it <= end and it % interval == 0 the u + p vector file
        <prefix>_000000_<it> (plus <prefix>_tavg_000000_<it> while averaging);
        finish_output() writes <prefix>.json and <prefix>.cv"""
        ctx = self.ctx
        self._out = {"prefix": str(prefix), "interval": int(interval), "start": start,
                     "end": end if end is not None else 1 << 62,
                     "tstart": tavg_start, "tend": tavg_end if tavg_end is not None else 1 << 62,
                     "fp64": as_fp64, "slices": [],
                     "uavg": ctx.field(3) if tavg_start is not None else None,
                     "pavg": ctx.field(1) if tavg_start is not None else None}

    def _output_step(self, o):
        it, ctx = self.it, self.ctx
        averaging = o["tstart"] is not None and o["tstart"] <= it <= o["tend"]
        if averaging:
            ctx.tavg(o["uavg"], self.u, it - o["tstart"] + 1)
            ctx.tavg(o["pavg"], self.p, it - o["tstart"] + 1)
        if o["start"] <= it <= o["end"] and it % o["interval"] == 0:
            ctx.write_vector_file(f"{o['prefix']}_{0:06d}_{it:010d}", [self.u, self.p], it, self.t(), o["fp64"])
            if averaging:
                ctx.write_vector_file(f"{o['prefix']}_tavg_{0:06d}_{it:010d}", [o["uavg"], o["pavg"]], it, self.t(), o["fp64"])
            o["slices"].append((it, self.t(), averaging))

    def finish_output(self):
        """wait for the queued snapshots, then the index and control-volume files"""
        from .api import write_index_file
        o = self._out
        self.ctx.io_wait()
        dsize = 8 if (o["fp64"] or self.ctx.precision == "fp64") else 4
        write_index_file(o["prefix"] + ".json", self.case.grid.interior, self.case.grid.gc, o["slices"], dsize)
        self.ctx.write_cv_file(o["prefix"] + ".cv")

    def snapshot(self):
        """keep a device copy of the state (fields and step counter) for restore()"""
        self._snap = ({k: getattr(self, k).clone() for k in ("u", "uu", "p", "nut")}, self.it)

    def restore(self):
        """return to the last snapshot (device-to-device copies on the current stream)"""
        fields, it = self._snap
        for k, v in fields.items():
            getattr(self, k).copy_(v)
        self.it = it

    def inlet_plane(self, it):
        """inlet velocity of step `it` sampled from the case's inflow box (as the
        library samples it): 3 x nz x ny, float64"""
        case = self.case
        box = case.inflow
        nx, ny, nz = case.grid.interior
        if box is None:
            plane = np.zeros((3, nz, ny))
            plane[0] = case.u_inlet
            return plane
        dx = float(case.grid.hx[case.grid.gc])
        xs = case.u_inlet * (it * case.dt) / dx
        fl = np.floor(xs)
        fr = xs - fl
        s0 = int(fl) % box.shape[1]
        s1 = (s0 + 1) % box.shape[1]
        plane = (1.0 - fr) * box[:, s0] + fr * box[:, s1]
        plane[0] += case.u_inlet
        return plane

    def state(self):
        import torch
        torch.cuda.synchronize()
        return {k: getattr(self, k).double().cpu().numpy() for k in ("u", "uu", "p", "nut")}

    def close(self):
        self.ctx.close()
