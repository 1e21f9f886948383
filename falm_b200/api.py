"""Python handle over the falm_b200 C ABI.

Method names follow the reference's solver classes (FalmCFD, FalmEq, FalmMV,
Alm::AlmHandler) so that a driver reads like app/nedo/main.cpp.  Fields are
torch CUDA tensors in the reference layout (component-major SoA over the
guide-cell box); torch is used for device memory and streams only, every
operation runs in this package's CUDA kernels.
"""
import ctypes
import numpy as np

from . import _lib as L


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _dp(a):
    return a.ctypes.data_as(L.c_double_p)


class Context:
    """One grid on one GPU (FalmCore without IO, src/falm.h:52-483)."""

    def __init__(self, grid, precision="fp64", device=None):
        import torch
        self.torch = torch
        self.lib = L.load()
        self.precision = precision
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.device = torch.device(device or "cuda:0")
        torch.cuda.set_device(self.device)
        self.grid = grid
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (grid.x, grid.y, grid.z, grid.hx, grid.hy, grid.hz)]
        g = L.Grid(grid.sx, grid.sy, grid.sz, grid.gc, *[_dp(a) for a in self._keep])
        h = ctypes.c_void_p()
        rc = self.lib.falm_create(ctypes.byref(g), L.FP64 if precision == "fp64" else L.MIXED, ctypes.byref(h))
        if rc != 0:
            raise L.FalmError(rc, "falm_create")
        self.h = h
        self.maxdiag = None
        self.alm_on = False

    # ------------------------------------------------------------ plumbing
    def _check(self, rc, where, allow=()):
        if rc != 0 and rc not in allow:
            raise L.FalmError(rc, where, self.lib.falm_last_error(self.h).decode())
        return rc

    def stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def close(self):
        if getattr(self, "h", None):
            self.lib.falm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, ncol=1):
        g = self.grid
        return self.torch.zeros(ncol * g.sx * g.sy * g.sz, dtype=self.dtype, device=self.device)

    def launches(self):
        return self.lib.falm_kernel_launches(self.h)

    # ------------------------------------------------------------ FalmCFD
    def cfd_init(self, Re, adv="Upwind3", sgs="Smagorinsky", Cs=0.1):
        self._check(self.lib.falm_cfd_init(self.h, Re, L.ADV[adv] if isinstance(adv, str) else adv,
                                           L.SGS[sgs] if isinstance(sgs, str) else sgs, Cs), "cfd_init")

    def pseudo_u(self, un, u, uu, ua, nut, ff, dt, t=0.0):
        self._check(self.lib.falm_cfd_pseudo_u(self.h, _ptr(un), _ptr(u), _ptr(uu), _ptr(ua), _ptr(nut), _ptr(ff),
                                               dt, t, self.stream()), "pseudo_u")

    def utouu(self, u, uu):
        self._check(self.lib.falm_cfd_utouu(self.h, _ptr(u), _ptr(uu), self.stream()), "utouu")

    def poisson_rhs(self, uu, rhs, dt, maxdiag):
        self._check(self.lib.falm_cfd_poisson_rhs(self.h, _ptr(uu), _ptr(rhs), dt, maxdiag, self.stream()), "rhs")

    def project_p(self, u, ua, uu, uua, p, dt):
        self._check(self.lib.falm_cfd_project_p(self.h, _ptr(u), _ptr(ua), _ptr(uu), _ptr(uua), _ptr(p), dt,
                                                self.stream()), "project_p")

    def sgs(self, u, nut):
        self._check(self.lib.falm_cfd_sgs(self.h, _ptr(u), _ptr(nut), self.stream()), "sgs")

    def divergence(self, uu, div):
        self._check(self.lib.falm_cfd_divergence(self.h, _ptr(uu), _ptr(div), self.stream()), "divergence")

    # ------------------------------------------------------------ FalmEq
    def eq_init(self, maxit, tol, pc="SOR", pc_maxit=2, pc_relax=1.2, ls="PBiCGStab", relax=1.0):
        self._check(self.lib.falm_eq_init(self.h, L.LS[ls], maxit, tol, relax, L.LS[pc], pc_maxit, pc_relax), "eq_init")

    def poisson_operator(self, bc_kind):
        md = ctypes.c_double()
        self._check(self.lib.falm_eq_poisson_operator(self.h, bc_kind, ctypes.byref(md)), "poisson_operator")
        self.maxdiag = md.value
        return md.value

    def set_matrix(self, A):
        self._A = A
        self._check(self.lib.falm_eq_set_matrix(self.h, _ptr(A)), "set_matrix")

    def solve(self, x, b, r):
        it, err = ctypes.c_int(), ctypes.c_double()
        rc = self._check(self.lib.falm_eq_solve(self.h, _ptr(x), _ptr(b), _ptr(r), self.stream(), ctypes.byref(it),
                                                ctypes.byref(err)), "solve", allow=(4, 5))
        return it.value, err.value, rc

    def res(self, x, b, r):
        self._check(self.lib.falm_eq_res(self.h, _ptr(x), _ptr(b), _ptr(r), self.stream()), "res")

    def sor_sweep(self, x, b, omega, color):
        self._check(self.lib.falm_eq_sor_sweep(self.h, _ptr(x), _ptr(b), omega, color, self.stream()), "sor")

    # ------------------------------------------------------------ FalmMV
    def mv(self, x, ax):
        self._check(self.lib.falm_mv_mv(self.h, _ptr(x), _ptr(ax), self.stream()), "mv")

    def dot(self, a, b):
        out = ctypes.c_double()
        self._check(self.lib.falm_mv_dot(self.h, _ptr(a), _ptr(b), ctypes.byref(out), self.stream()), "dot")
        return out.value

    def normsq(self, a, ncol=1):
        out = ctypes.c_double()
        self._check(self.lib.falm_mv_normsq(self.h, _ptr(a), ncol, ctypes.byref(out), self.stream()), "normsq")
        return out.value

    def maxdiag_of(self):
        out = ctypes.c_double()
        self._check(self.lib.falm_mv_maxdiag(self.h, ctypes.byref(out)), "maxdiag")
        return out.value

    def scale(self, a, s):
        self._check(self.lib.falm_mv_scale(self.h, _ptr(a), a.numel(), s, self.stream()), "scale")

    def axby(self, a, x, b, y, out):
        self._check(self.lib.falm_mv_axby(self.h, a, _ptr(x), b, _ptr(y), _ptr(out), x.numel(), self.stream()), "axby")

    # ------------------------------------------------------------ boundary conditions
    def bc_init(self, kind, u_inlet=1.0):
        self._check(self.lib.falm_bc_init(self.h, kind, u_inlet), "bc_init")

    def set_inflow(self, box, dx):
        if box is None:
            self._check(self.lib.falm_bc_set_inflow(self.h, None, 0, 0.0), "set_inflow")
            return
        box = np.ascontiguousarray(box, dtype=np.float64)
        self._check(self.lib.falm_bc_set_inflow(self.h, _dp(box), box.shape[1], dx), "set_inflow")

    def ubc(self, u, uprev, dt, t):
        self._check(self.lib.falm_bc_ubc(self.h, _ptr(u), _ptr(uprev), dt, t, self.stream()), "ubc")

    def pbc(self, p):
        self._check(self.lib.falm_bc_pbc(self.h, _ptr(p), self.stream()), "pbc")

    def uubc(self, uu):
        self._check(self.lib.falm_bc_uubc(self.h, _ptr(uu), self.stream()), "uubc")

    # ------------------------------------------------------------ ALM
    def alm_init(self, alm):
        """alm: falm_b200.cases.AlmSetup"""
        self._alm_keep = alm.arrays()
        k = self._alm_keep
        d = L.AlmDesc(alm.n_turbine, alm.n_blade, alm.n_ap_per_blade, alm.n_attack, alm.radius, alm.hub_radius,
                      alm.euler_eps, _dp(k["base"]), _dp(k["hub"]), _dp(k["tip_rate"]), _dp(k["motion"]),
                      k["angle_type"].ctypes.data_as(L.c_int_p), _dp(k["ap_r"]), _dp(k["ap_chord"]),
                      _dp(k["ap_twist"]), _dp(k["attack"]), _dp(k["cl"]), _dp(k["cd"]), alm.pitch)
        self._check(self.lib.falm_alm_init(self.h, ctypes.byref(d)), "alm_init")
        self.alm_on = True
        self.n_turbine = alm.n_turbine

    def set_pitch(self, deg):
        self._check(self.lib.falm_alm_set_pitch(self.h, deg), "set_pitch")

    def alm_run(self, u, ff, t):
        tq = np.zeros(self.n_turbine)
        th = np.zeros(self.n_turbine)
        self._check(self.lib.falm_alm_run(self.h, _ptr(u), _ptr(ff), t, self.stream(), _dp(tq), _dp(th)), "alm_run")
        return tq, th

    def alm_aps(self, apcount):
        xyz, f = np.zeros(3 * apcount), np.zeros(3 * apcount)
        tq, th = np.zeros(apcount), np.zeros(apcount)
        self._check(self.lib.falm_alm_get_aps(self.h, _dp(xyz), _dp(f), _dp(tq), _dp(th)), "alm_get_aps")
        return xyz.reshape(apcount, 3), f.reshape(apcount, 3), tq, th

    def set_inlet_plane(self, plane_pinned):
        """plane: pinned host float64 tensor/array 3 x nz x ny (interior), used by the next
        velocity BC (the next step), which copies it: keep it alive and unchanged until then"""
        ptr = ctypes.cast(ctypes.c_void_p(plane_pinned.data_ptr()), L.c_double_p)
        self._check(self.lib.falm_bc_set_inlet_plane(self.h, ptr, self.stream()), "set_inlet_plane")

    # ------------------------------------------------------------ instrumentation
    def profile(self, enable=True):
        self._check(self.lib.falm_profile_enable(self.h, 1 if enable else 0), "profile_enable")

    def profile_read(self, reset=True):
        n = len(L.KERNEL_CLASSES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        self._check(self.lib.falm_profile_read(self.h, ms, cnt, n, 1 if reset else 0), "profile_read")
        return {k: (ms[i], cnt[i]) for i, k in enumerate(L.KERNEL_CLASSES)}

    # ------------------------------------------------------------ step
    def step(self, u, uu, p, nut, ff, dt, t):
        fl = L.Fields(_ptr(u), _ptr(uu), _ptr(p), _ptr(nut), _ptr(ff))
        st = L.StepStats()
        self._check(self.lib.falm_step(self.h, ctypes.byref(fl), dt, t, self.stream(), ctypes.byref(st)), "step")
        n = getattr(self, "n_turbine", 0)
        return {"it": st.it, "err": st.err, "divnorm": st.divnorm, "outer": st.outer, "status": st.status,
                "torque": list(st.torque[:n]), "thrust": list(st.thrust[:n])}

    def step_adjoint(self, u, uu, p, nut, dt, t, w_power, au, auu, anut, grad, u_after=None):
        """falm_step_adjoint: maps the adjoint of the state after the step (au, auu,
        anut, in place) to the state before it and adds the step's gradient into grad;
        u_after (the velocity after the step) spares the recomputation of the step"""
        fl = L.Fields(_ptr(u), _ptr(uu), _ptr(p), _ptr(nut), None)
        f1 = L.Fields(_ptr(u_after), None, None, None, None) if u_after is not None else None
        self._check(self.lib.falm_step_adjoint(self.h, ctypes.byref(fl), ctypes.byref(f1) if f1 is not None else None, dt, t,
                                               w_power, _ptr(au), _ptr(auu), _ptr(anut), _ptr(grad), self.stream()),
                    "step_adjoint")


    # ------------------------------------------------------------ RMCP rotor model
    def rmcp_init(self, r):
        """Rmcp::RmcpAlm::init from a cases.RmcpSetup: the step's forcing becomes the RMCP model"""
        k = r.arrays()
        self._rmcp_keep = k
        d = L.RmcpDesc(r.n_turbine, r.n_blade, r.radius, r.hub_radius, r.width, r.thick, _dp(k["base"]), _dp(k["hub"]),
                       _dp(k["angle"]), k["angle_type"].ctypes.data_as(L.c_int_p), _dp(k["tip_rate"]), len(k["st_r"]),
                       len(k["attack"]), _dp(k["st_r"]), _dp(k["st_chord"]), _dp(k["st_twist"]), _dp(k["attack"]),
                       _dp(k["cl"]), _dp(k["cd"]))
        self._check(self.lib.falm_rmcp_init(self.h, ctypes.byref(d)), "rmcp_init")
        self.n_turbine = r.n_turbine
        self.alm_on = False

    def rmcp_run(self, u, ff, t, flag=None):
        """SetALMFlag + ALM of the RMCP model at time t into ff (and the paint into the int32
        device tensor flag); returns per-turbine torque and thrust"""
        n = self.n_turbine
        tq, th = np.zeros(n), np.zeros(n)
        self._check(self.lib.falm_rmcp_run(self.h, _ptr(u), _ptr(ff), t, self.stream(), _ptr(flag), _dp(tq), _dp(th)),
                    "rmcp_run")
        return tq, th

    # ------------------------------------------------------------ z slabs
    def slab_init(self, rank, nranks, z_offset, nz_global, transport):
        """falm_slab_init: this context is slab `rank` of a grid split along z"""
        self._transport = transport
        self._check(self.lib.falm_slab_init(self.h, rank, nranks, z_offset, nz_global, ctypes.byref(transport)), "slab_init")

    def slab_halo(self, field, depth=1):
        """exchange `depth` guide planes of a field with the neighbouring slabs"""
        ncol = field.numel() // self.grid.n
        self._check(self.lib.falm_slab_halo(self.h, _ptr(field), ncol, depth, self.stream()), "slab_halo")

    def adjoint_set_tol(self, rel_tol):
        """relative residual of the adjoint's transposed Poisson solve (0: the default)"""
        self._check(self.lib.falm_adjoint_set_tol(self.h, float(rel_tol)), "adjoint_set_tol")

    # ------------------------------------------------------------ output (FalmIO, TAvg)
    def tavg(self, avg, f, count):
        """FalmSolver::TAvg (src/falm.h:433-444): avg = (1 - 1/count) avg + f/count"""
        ncol = f.numel() // self.grid.n
        self._check(self.lib.falm_tavg(self.h, _ptr(avg), _ptr(f), ncol, count, self.stream()), "tavg")

    def write_vector_file(self, path, fields, step, time, as_fp64=False):
        """FalmIO::writeVectorFile of the columns of `fields` (device tensors) in order;
        returns before the file is written (see io_wait)"""
        ptrs = (L.P * len(fields))(*[f.data_ptr() for f in fields])
        ncols = (ctypes.c_int * len(fields))(*[f.numel() // self.grid.n for f in fields])
        self._check(self.lib.falm_io_write_vector_file(self.h, str(path).encode(), ptrs, ncols, len(fields), int(step),
                                                       float(time), 1 if as_fp64 else 0, self.stream()),
                    "write_vector_file")

    def read_vector_file(self, path, fields):
        """the inverse of write_vector_file: the file's columns into `fields` (device
        tensors, in order); returns (step, time) of its header"""
        ptrs = (L.P * len(fields))(*[f.data_ptr() for f in fields])
        ncols = (ctypes.c_int * len(fields))(*[f.numel() // self.grid.n for f in fields])
        step, time = ctypes.c_ulonglong(), ctypes.c_double()
        self._check(self.lib.falm_io_read_vector_file(self.h, str(path).encode(), ptrs, ncols, len(fields), ctypes.byref(step),
                                                      ctypes.byref(time), self.stream()), "read_vector_file")
        return step.value, time.value

    def io_wait(self):
        """wait for every queued snapshot file"""
        self._check(self.lib.falm_io_wait(self.h), "io_wait")

    def write_cv_file(self, path):
        """FalmIO::writeControlVolumeFile of this grid"""
        self._check(self.lib.falm_io_write_cv_file(self.h, str(path).encode()), "write_cv_file")


def write_index_file(path, interior, gc, snapshots, dsize=8):
    """FalmIO::writeIndexFile (src/FalmIO.h:25-67); snapshots: [(step, time, tavg), ...]"""
    lib = L.load()
    n = len(snapshots)
    steps = (ctypes.c_ulonglong * max(n, 1))(*[int(s[0]) for s in snapshots])
    times = np.ascontiguousarray([float(s[1]) for s in snapshots] or [0.0], dtype=np.float64)
    tav = (ctypes.c_int * max(n, 1))(*[1 if s[2] else 0 for s in snapshots])
    rc = lib.falm_io_write_index_file(str(path).encode(), interior[0], interior[1], interior[2], gc, steps, _dp(times),
                                      tav, n, dsize)
    if rc != 0:
        raise L.FalmError(rc, "write_index_file")


def read_cv_file(path):
    """FalmIO::readControlVolumeFile (src/FalmIO.h:99-116): (dims (sx, sy, sz, gc), x, hx, y, hy, z, hz)"""
    lib = L.load()
    dims = (ctypes.c_int * 4)()
    rc = lib.falm_io_read_cv_file(str(path).encode(), dims, None, None, None, None, None, None)
    if rc != 0:
        raise L.FalmError(rc, "read_cv_file")
    arr = [np.zeros(dims[d // 2]) for d in range(6)]
    rc = lib.falm_io_read_cv_file(str(path).encode(), dims, *[_dp(a) for a in arr])
    if rc != 0:
        raise L.FalmError(rc, "read_cv_file")
    return tuple(dims), arr[0], arr[1], arr[2], arr[3], arr[4], arr[5]


def build_mesh(cvcenter, meshpath, outputfile, gc=2):
    """Mesher::build_mesh (src/mesher/mesher.hpp:12-260): a control-volume file from node coordinates"""
    rc = L.load().falm_mesh_build(cvcenter.encode(), str(meshpath).encode(), str(outputfile).encode(), gc)
    if rc != 0:
        raise L.FalmError(rc, "build_mesh")


def read_vector_file(path):
    """a FalmIO vector file: (header dict, array [ncol, kmax, jmax, imax])"""
    with open(path, "rb") as f:
        head = np.frombuffer(f.read(48), dtype=np.uint64)
        time = np.frombuffer(f.read(8), dtype=np.float64)[0]
        dsize = int(np.frombuffer(f.read(8), dtype=np.uint64)[0])
        imax, jmax, kmax, ncol, gc, step = (int(v) for v in head)
        data = np.frombuffer(f.read(), dtype=np.float64 if dsize == 8 else np.float32)
    hd = {"imax": imax, "jmax": jmax, "kmax": kmax, "ncol": ncol, "gc": gc, "step": step, "time": float(time), "dsize": dsize}
    return hd, data.reshape(ncol, kmax, jmax, imax)


def build_aps(stations, n_turbine, n_blade, n_ap_per_blade, radius, hub_radius):
    """BladeHandler::buildAP (src/alm/bladeHandler.h:16-104) through the C ABI (host only)."""
    lib = L.load()
    st_r = np.ascontiguousarray(stations["r"], dtype=np.float64)
    st_c = np.ascontiguousarray(stations["chord"], dtype=np.float64)
    st_t = np.ascontiguousarray(stations["twist"], dtype=np.float64)
    st_cl = np.ascontiguousarray(stations["cl"], dtype=np.float64)
    st_cd = np.ascontiguousarray(stations["cd"], dtype=np.float64)
    na = st_cl.shape[1]
    apc = n_turbine * n_blade * n_ap_per_blade
    out = {k: np.zeros(apc) for k in ("r", "chord", "twist")}
    cl, cd = np.zeros(apc * na), np.zeros(apc * na)
    rc = lib.falm_alm_build_aps(len(st_r), _dp(st_r), _dp(st_c), _dp(st_t), _dp(st_cl), _dp(st_cd), na, apc,
                                n_ap_per_blade, radius, hub_radius, _dp(out["r"]), _dp(out["chord"]),
                                _dp(out["twist"]), _dp(cl), _dp(cd))
    if rc != 0:
        raise L.FalmError(rc, "build_aps")
    out["cl"], out["cd"] = cl, cd
    return out
