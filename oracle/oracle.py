"""ctypes binding of the CPU oracle (liboracle.so) and of the reference's own
CUDA step (oracle/_ref/libfalmref.so).  Test infrastructure only: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
product package.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfalmref.so")
dp = ctypes.POINTER(ctypes.c_double)
ip = ctypes.POINTER(ctypes.c_int)

RF = dict(U=0, UU=1, P=2, NUT=3, FF=4, RHS=5, RES=6, UPREV=7, DIV=8, A=9, KX=10, G=11, JA=12)
RO = dict(PSEUDO_U=0, UTOUU=1, RHS=2, SOLVE=3, PBC=4, PROJECT=5, UBC=6, SGS=7, DIV=8, ALM=9, UUBC=10)
ADV = {"Upwind1": 0, "Upwind3": 1, "QUICK": 2, "UTOPIA": 3, "KK": 4}
SGS = {"Empty": 0, "Smagorinsky": 1, "CSM": 2}
PC = {"None": 0, "Jacobi": 1, "SOR": 2}


class OrAlm(ctypes.Structure):
    _fields_ = [("n_turbine", ctypes.c_int), ("n_blade", ctypes.c_int), ("n_ap_per_blade", ctypes.c_int),
                ("n_attack", ctypes.c_int), ("radius", ctypes.c_double), ("hub_radius", ctypes.c_double),
                ("euler_eps", ctypes.c_double), ("base", dp), ("hub", dp), ("tip_rate", dp), ("motion", dp),
                ("angle_type", ip), ("ap_r", dp), ("ap_chord", dp), ("ap_twist", dp), ("attack", dp),
                ("cl", dp), ("cd", dp), ("pitch", ctypes.c_double)]


class OrRmcp(ctypes.Structure):
    _fields_ = [("n_turbine", ctypes.c_int), ("n_blade", ctypes.c_int), ("radius", ctypes.c_double),
                ("hub_radius", ctypes.c_double), ("width", ctypes.c_double), ("thick", ctypes.c_double),
                ("base", dp), ("hub", dp), ("angle", dp), ("angle_type", ip), ("tip_rate", dp),
                ("n_station", ctypes.c_int), ("n_attack", ctypes.c_int), ("st_r", dp), ("st_chord", dp),
                ("st_twist", dp), ("attack", dp), ("cl", dp), ("cd", dp)]


def rmcp_struct(r):
    """an or_rmcp for a cases.RmcpSetup (and the arrays it points into)"""
    k = r.arrays()
    s = OrRmcp(r.n_turbine, r.n_blade, r.radius, r.hub_radius, r.width, r.thick, _p(k["base"]), _p(k["hub"]),
               _p(k["angle"]), k["angle_type"].ctypes.data_as(ip), _p(k["tip_rate"]), len(k["st_r"]), len(k["attack"]),
               _p(k["st_r"]), _p(k["st_chord"]), _p(k["st_twist"]), _p(k["attack"]), _p(k["cl"]), _p(k["cd"]))
    return s, k


class OrCase(ctypes.Structure):
    _fields_ = [("sx", ctypes.c_int), ("sy", ctypes.c_int), ("sz", ctypes.c_int), ("gc", ctypes.c_int),
                ("x", dp), ("hx", dp), ("y", dp), ("hy", dp), ("z", dp), ("hz", dp),
                ("Re", ctypes.c_double), ("Cs", ctypes.c_double), ("dt", ctypes.c_double),
                ("adv", ctypes.c_int), ("sgs", ctypes.c_int),
                ("ls_maxit", ctypes.c_int), ("ls_tol", ctypes.c_double), ("pc_type", ctypes.c_int),
                ("pc_maxit", ctypes.c_int), ("pc_relax", ctypes.c_double),
                ("bc", ctypes.c_int), ("u_inlet", ctypes.c_double),
                ("inflow_box", dp), ("inflow_nb", ctypes.c_int), ("inflow_dx", ctypes.c_double),
                ("alm_on", ctypes.c_int), ("alm", OrAlm)]


class OrStats(ctypes.Structure):
    _fields_ = [("it", ctypes.c_int), ("err", ctypes.c_double), ("divnorm", ctypes.c_double),
                ("torque", ctypes.c_double * 8), ("thrust", ctypes.c_double * 8)]


def _p(a):
    return None if a is None else a.ctypes.data_as(dp)


def build(ref=False):
    """Compile the oracle; with ref=True also oracle/_ref when the recipe finds the
    reference's sources (FALM_REFERENCE, see oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)


class CaseStruct:
    """Holds an or_case and the numpy arrays it points into."""

    def __init__(self, case, use_inflow=True, maxit=None, tol=None):
        g = case.grid
        self.keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (g.x, g.hx, g.y, g.hy, g.z, g.hz)]
        c = OrCase()
        c.sx, c.sy, c.sz, c.gc = g.sx, g.sy, g.sz, g.gc
        c.x, c.hx, c.y, c.hy, c.z, c.hz = [_p(a) for a in self.keep]
        c.Re, c.Cs, c.dt = case.Re, case.Cs, case.dt
        c.adv, c.sgs = ADV[case.adv], SGS[case.sgs]
        c.ls_maxit = case.maxit if maxit is None else maxit
        c.ls_tol = case.tol if tol is None else tol
        c.pc_type, c.pc_maxit, c.pc_relax = PC[case.pc], case.pc_maxit, case.pc_relax
        c.bc, c.u_inlet = case.bc, case.u_inlet
        if use_inflow and case.inflow is not None:
            self.inflow = np.ascontiguousarray(case.inflow, dtype=np.float64)
            c.inflow_box, c.inflow_nb, c.inflow_dx = _p(self.inflow), self.inflow.shape[1], float(g.hx[g.gc])
        else:
            c.inflow_box, c.inflow_nb, c.inflow_dx = None, 0, 1.0
        c.alm_on = 0
        if case.alm is not None:
            a = case.alm
            self.alm_arrays = a.arrays()
            k = self.alm_arrays
            c.alm_on = 1
            c.alm = OrAlm(a.n_turbine, a.n_blade, a.n_ap_per_blade, a.n_attack, a.radius, a.hub_radius, a.euler_eps,
                          _p(k["base"]), _p(k["hub"]), _p(k["tip_rate"]), _p(k["motion"]),
                          k["angle_type"].ctypes.data_as(ip), _p(k["ap_r"]), _p(k["ap_chord"]), _p(k["ap_twist"]),
                          _p(k["attack"]), _p(k["cl"]), _p(k["cd"]), a.pitch)
        self.c = c
        self.case = case


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        self.L = L
        P, C, D, I = ctypes.c_void_p, ctypes.POINTER(OrCase), ctypes.c_double, ctypes.c_int
        sig = {
            "oracle_metrics": [C, dp, dp, dp], "oracle_poisson_matrix": [C, dp, dp, dp],
            "oracle_pseudo_u": [C, dp, dp, dp, dp, dp, dp, dp, dp, dp], "oracle_utouu": [C, dp, dp, dp, dp],
            "oracle_divergence": [C, dp, dp, dp], "oracle_poisson_rhs": [C, dp, dp, dp, D],
            "oracle_project_p": [C, dp, dp, dp, dp, dp, dp, dp], "oracle_sgs": [C, dp, dp, dp, dp],
            "oracle_mv": [C, dp, dp, dp], "oracle_dot": [C, dp, dp], "oracle_normsq": [C, dp, I],
            "oracle_res": [C, dp, dp, dp, dp], "oracle_sor_sweep": [C, dp, dp, dp, D, I],
            "oracle_pbicgstab": [C, dp, dp, dp, dp, ip, dp], "oracle_ubc": [C, dp, dp, D],
            "oracle_plain_solve": [C, I, D, dp, dp, dp, dp, ip, dp],
            "oracle_pbc": [C, dp], "oracle_uubc": [C, dp],
            "oracle_build_aps": [I, dp, dp, dp, dp, dp, I, I, I, D, D, dp, dp, dp, dp, dp],
            "oracle_alm": [C, dp, dp, D, dp, dp, dp, dp, dp, dp],
            "oracle_step": [C, dp, dp, dp, dp, dp, dp, dp, dp, dp, D, D, ctypes.POINTER(OrStats)],
            "oracle_num_threads": [],
            "oracle_transpose_matrix": [C, dp, dp],
            "oracle_step_adjoint": [C, dp, dp, dp, dp, dp, dp, dp, dp, dp, D, D, D, dp, dp, dp, dp, dp, dp],
            "oracle_rmcp": [C, ctypes.POINTER(OrRmcp), dp, dp, ip, D, dp, dp],
        }
        for k, v in sig.items():
            getattr(L, k).argtypes = v
            getattr(L, k).restype = ctypes.c_int
        for k in ("oracle_poisson_matrix", "oracle_dot", "oracle_normsq"):
            getattr(L, k).restype = ctypes.c_double
        for k in ("oracle_metrics", "oracle_pseudo_u", "oracle_utouu", "oracle_divergence", "oracle_poisson_rhs",
                  "oracle_project_p", "oracle_sgs", "oracle_mv", "oracle_res", "oracle_sor_sweep",
                  "oracle_pbicgstab", "oracle_plain_solve", "oracle_ubc", "oracle_pbc", "oracle_uubc", "oracle_build_aps",
                  "oracle_alm", "oracle_step", "oracle_transpose_matrix", "oracle_rmcp"):
            getattr(L, k).restype = None

    def threads(self):
        return self.L.oracle_num_threads()

    def setup(self, cs):
        """metrics + Poisson matrix for a CaseStruct; returns dict"""
        n = cs.case.grid.n
        kx, g, ja, A = np.zeros(3 * n), np.zeros(3 * n), np.zeros(n), np.zeros(7 * n)
        self.L.oracle_metrics(ctypes.byref(cs.c), _p(kx), _p(g), _p(ja))
        md = self.L.oracle_poisson_matrix(ctypes.byref(cs.c), _p(g), _p(ja), _p(A))
        return {"kx": kx, "g": g, "ja": ja, "A": A, "maxdiag": md}

    def step(self, cs, st, m, t):
        """one step in place on the state dict st (u, uu, p, nut, ff)"""
        s = OrStats()
        self.L.oracle_step(ctypes.byref(cs.c), _p(st["u"]), _p(st["uu"]), _p(st["p"]), _p(st["nut"]), _p(st["ff"]),
                           _p(m["kx"]), _p(m["g"]), _p(m["ja"]), _p(m["A"]), m["maxdiag"], t, ctypes.byref(s))
        n = cs.c.alm.n_turbine if cs.c.alm_on else 0
        return {"it": s.it, "err": s.err, "divnorm": s.divnorm, "torque": list(s.torque[:n]), "thrust": list(s.thrust[:n])}

    def init_state(self, cs, m, st):
        """UtoUU and SGS at start (app/nedo/main.cpp:132-133)"""
        c = ctypes.byref(cs.c)
        self.L.oracle_utouu(c, _p(st["u"]), _p(st["uu"]), _p(m["kx"]), _p(m["ja"]))
        self.L.oracle_sgs(c, _p(st["u"]), _p(st["nut"]), _p(m["kx"]), _p(m["ja"]))

    def pbicgstab(self, cs, A, x, b, r):
        it, err = ctypes.c_int(), ctypes.c_double()
        self.L.oracle_pbicgstab(ctypes.byref(cs.c), _p(A), _p(x), _p(b), _p(r), ctypes.byref(it), ctypes.byref(err))
        return it.value, err.value

    def plain_solve(self, cs, ls, relax, A, x, b, r):
        """FalmEq::Jacobi / FalmEq::SOR (ls "Jacobi" or "SOR") with the case's maxit and tol"""
        it, err = ctypes.c_int(), ctypes.c_double()
        self.L.oracle_plain_solve(ctypes.byref(cs.c), PC[ls], relax, _p(A), _p(x), _p(b), _p(r), ctypes.byref(it),
                                  ctypes.byref(err))
        return it.value, err.value

    def power(self, cs, stats):
        """rotor power of a step: sum over turbines of torque * tip rate (src/alm/alm.h:133)"""
        tip = cs.alm_arrays["tip_rate"]
        return float(sum(tq * tr for tq, tr in zip(stats["torque"], tip)))

    def objective(self, cs, m, st0, steps, it0):
        """J = mean rotor power over `steps` steps from state st0 (step n at time (it0 + n) dt)"""
        st = {k: v.copy() for k, v in st0.items()}
        J = 0.0
        for q in range(steps):
            J += self.power(cs, self.step(cs, st, m, (it0 + q + 1) * cs.case.dt)) / steps
        return J

    def adjoint(self, cs, m, st0, steps, it0):
        """J and its gradient with respect to (collective pitch, per-AP chord, per-AP
        twist) by the discrete adjoint of the steps (all states kept in memory)"""
        c = ctypes.byref(cs.c)
        n = cs.case.grid.n
        AT = np.zeros(7 * n)
        self.L.oracle_transpose_matrix(c, _p(m["A"]), _p(AT))
        st = {k: v.copy() for k, v in st0.items()}
        states, J = [], 0.0
        for q in range(steps):
            states.append({k: st[k].copy() for k in ("u", "uu", "nut", "p")})
            J += self.power(cs, self.step(cs, st, m, (it0 + q + 1) * cs.case.dt)) / steps
        a = cs.c.alm
        apc = a.n_turbine * a.n_blade * a.n_ap_per_blade
        gp, gch, gtw = np.zeros(1), np.zeros(apc), np.zeros(apc)
        au, auu, anut = np.zeros(3 * n), np.zeros(3 * n), np.zeros(n)
        for q in reversed(range(steps)):
            S = states[q]
            rc = self.L.oracle_step_adjoint(c, _p(S["u"]), _p(S["uu"]), _p(S["nut"]), _p(S["p"]), _p(m["kx"]), _p(m["g"]),
                                            _p(m["ja"]), _p(m["A"]), _p(AT), m["maxdiag"], (it0 + q + 1) * cs.case.dt,
                                            1.0 / steps, _p(au), _p(auu), _p(anut), _p(gp), _p(gch), _p(gtw))
            if rc:
                raise ValueError("oracle_step_adjoint: unsupported scheme or SGS model")
        return J, float(gp[0]), gch, gtw

    def rmcp(self, cs, r, u, t):
        """oracle_rmcp: force field, paint, per-turbine torque and thrust of the RMCP model"""
        rs, keep = rmcp_struct(r)
        n = cs.case.grid.n
        ff, flag = np.zeros(3 * n), np.zeros(n, dtype=np.int32)
        tq, th = np.zeros(r.n_turbine), np.zeros(r.n_turbine)
        self.L.oracle_rmcp(ctypes.byref(cs.c), ctypes.byref(rs), _p(u), _p(ff), flag.ctypes.data_as(ip), t, _p(tq), _p(th))
        return ff, flag, tq, th

    def alm(self, cs, u, ff, t):
        a = cs.c.alm
        apc = a.n_turbine * a.n_blade * a.n_ap_per_blade
        xyz, f, tq, th = np.zeros(3 * apc), np.zeros(3 * apc), np.zeros(apc), np.zeros(apc)
        ttq, tth = np.zeros(a.n_turbine), np.zeros(a.n_turbine)
        self.L.oracle_alm(ctypes.byref(cs.c), _p(u), _p(ff), t, _p(xyz), _p(f), _p(tq), _p(th), _p(ttq), _p(tth))
        return {"xyz": xyz.reshape(apc, 3), "force": f.reshape(apc, 3), "torque_ap": tq, "thrust_ap": th,
                "torque": ttq, "thrust": tth}


class RefStep:
    """The reference's own CUDA step (oracle/_ref/libfalmref.so), on the GPU."""

    def __init__(self, cs, workdir):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        L = ctypes.CDLL(REF_SO)
        self.L = L
        P = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.POINTER(OrCase), ctypes.c_int, dp, dp, dp, dp, dp, ctypes.c_char_p]
        L.ref_create.restype = P
        L.ref_destroy.argtypes = [P]
        L.ref_destroy.restype = None
        L.ref_maxdiag.argtypes = [P]
        L.ref_maxdiag.restype = ctypes.c_double
        L.ref_set.argtypes = [P, ctypes.c_int, dp]
        L.ref_get.argtypes = [P, ctypes.c_int, dp]
        L.ref_op.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.POINTER(OrStats)]
        L.ref_step.argtypes = [P, ctypes.c_double, ctypes.POINTER(OrStats)]
        L.ref_get_aps.argtypes = [P, dp, dp, dp, dp]
        L.ref_plain_solve.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.POINTER(OrStats)]
        L.ref_write_uvwp.argtypes = [P, ctypes.c_char_p, ctypes.c_ulonglong, ctypes.c_double]
        L.ref_write_index.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_ulonglong), dp,
                                      ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.ref_write_cv.argtypes = [P, ctypes.c_char_p]
        L.ref_rmcp_init.argtypes = [P, ctypes.POINTER(OrRmcp)]
        L.ref_rmcp_run.argtypes = [P, ctypes.c_double, dp, ip]
        self.cs = cs
        self.n = cs.case.grid.n
        st = cs.case.alm.stations if cs.case.alm is not None else None
        if st is not None:
            self.st = {k: np.ascontiguousarray(st[k], dtype=np.float64) for k in ("r", "chord", "twist", "cl", "cd")}
            args = [len(self.st["r"]), _p(self.st["r"]), _p(self.st["chord"]), _p(self.st["twist"]),
                    _p(self.st["cl"]), _p(self.st["cd"])]
        else:
            args = [0, None, None, None, None, None]
        os.makedirs(workdir, exist_ok=True)
        self.h = L.ref_create(ctypes.byref(cs.c), *args, workdir.encode())
        if not self.h:
            raise RuntimeError("ref_create failed")

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def ncol(self, fid):
        return {RF["U"]: 3, RF["UU"]: 3, RF["FF"]: 3, RF["UPREV"]: 3, RF["A"]: 7, RF["KX"]: 3, RF["G"]: 3}.get(fid, 1)

    def set(self, name, arr):
        fid = RF[name]
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.size == self.ncol(fid) * self.n
        rc = self.L.ref_set(self.h, fid, _p(a))
        if rc:
            raise RuntimeError(f"ref_set {name}: {rc}")

    def get(self, name):
        fid = RF[name]
        a = np.zeros(self.ncol(fid) * self.n)
        rc = self.L.ref_get(self.h, fid, _p(a))
        if rc:
            raise RuntimeError(f"ref_get {name}: {rc}")
        return a

    def op(self, name, t=0.0):
        s = OrStats()
        rc = self.L.ref_op(self.h, RO[name], t, ctypes.byref(s))
        if rc:
            raise RuntimeError(f"ref_op {name}: {rc}")
        return s

    def step(self, t):
        s = OrStats()
        rc = self.L.ref_step(self.h, t, ctypes.byref(s))
        if rc:
            raise RuntimeError(f"ref_step: {rc}")
        n = self.cs.c.alm.n_turbine if self.cs.c.alm_on else 0
        return {"it": s.it, "err": s.err, "divnorm": s.divnorm, "torque": list(s.torque[:n]), "thrust": list(s.thrust[:n])}

    def maxdiag(self):
        return self.L.ref_maxdiag(self.h)

    def plain_solve(self, ls, relax, maxit, tol):
        """FalmEq::Solve with the plain Jacobi / SOR solver on the harness's P, RHS, RES"""
        s = OrStats()
        rc = self.L.ref_plain_solve(self.h, PC[ls], relax, maxit, tol, ctypes.byref(s))
        if rc:
            raise RuntimeError(f"ref_plain_solve: {rc}")
        return s.it, s.err

    def write_uvwp(self, path, step, time):
        """FalmIO::writeVectorFile of u and p, as the drivers' outputUVWP"""
        rc = self.L.ref_write_uvwp(self.h, str(path).encode(), int(step), float(time))
        if rc:
            raise RuntimeError(f"ref_write_uvwp: {rc}")

    def write_index(self, path, snapshots):
        """FalmIO::writeIndexFile; snapshots: [(step, time, tavg), ...]"""
        n = len(snapshots)
        steps = (ctypes.c_ulonglong * max(n, 1))(*[int(q[0]) for q in snapshots])
        times = np.ascontiguousarray([float(q[1]) for q in snapshots] or [0.0])
        tav = (ctypes.c_int * max(n, 1))(*[1 if q[2] else 0 for q in snapshots])
        self.L.ref_write_index(self.h, str(path).encode(), steps, _p(times), tav, n)

    def rmcp_init(self, r):
        """the reference's RmcpAlm::init for a cases.RmcpSetup"""
        self._rmcp = rmcp_struct(r)
        rc = self.L.ref_rmcp_init(self.h, ctypes.byref(self._rmcp[0]))
        if rc:
            raise RuntimeError(f"ref_rmcp_init: {rc}")

    def rmcp_run(self, t):
        """RmcpAlm::SetALMFlag + ALM on the harness's U: (ff, flag)"""
        ff, flag = np.zeros(3 * self.n), np.zeros(self.n, dtype=np.int32)
        rc = self.L.ref_rmcp_run(self.h, t, _p(ff), flag.ctypes.data_as(ip))
        if rc:
            raise RuntimeError(f"ref_rmcp_run: {rc}")
        return ff, flag

    def write_cv(self, path):
        """FalmIO::writeControlVolumeFile of the case grid"""
        self.L.ref_write_cv(self.h, str(path).encode())
