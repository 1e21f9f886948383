"""Synthetic cases of the LES step (grids, turbine, polars, seeded inflow).

Lengths are in rotor radii (R = 1) and the inflow velocity is U = 1: the
reference's actuator-point tables are only self-consistent at R = 1 (its
BladeHandler stores chord/R as chord, src/alm/bladeHandler.h:32,51-57,76).

Cases (the grid is the interior size; two guide cells on every side):
  cavity  64^3 lid-driven cavity, Re 1000, dt 1e-3, Cs 0.1, Upwind3,
          PBiCGStab + red-black SOR (2 sweeps, omega 1.2), tol 1e-8
  channel 256x128x128, h = 1/20 (R = 20 cells), one 3-blade rotor (TSR 7,
          32 points per blade), Gaussian width 2h, synthetic polars,
          seeded 5% inflow, Re 1e4, dt = 0.3 h, tol 1e-8
  channel_large 512x256x256 with the same physics and h, tol 1e-6
  adjoint 128x64x64, R = 10 cells
  floating 1024x256x256, R = 24 cells, TSR 9, blade pitch 3 deg,
          platform pitch 3 deg sin(2 pi t / 10), 8% inflow
"""
from dataclasses import dataclass, field
import math
import numpy as np

GC = 2
INFLOW_SEED = 20261203


@dataclass
class Grid:
    sx: int
    sy: int
    sz: int
    gc: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    hx: np.ndarray
    hy: np.ndarray
    hz: np.ndarray

    @property
    def n(self):
        return self.sx * self.sy * self.sz

    @property
    def interior(self):
        return (self.sx - 2 * self.gc, self.sy - 2 * self.gc, self.sz - 2 * self.gc)

    @property
    def n_interior(self):
        a, b, c = self.interior
        return a * b * c


def uniform_grid(nx, ny, nz, h, gc=GC, origin=(0.0, 0.0, 0.0)):
    """Control volumes centred at origin + (i+1/2)h, i = -gc..n+gc-1 (app/lid3d/cv.py:9-22)."""
    def axis(n, o):
        i = np.arange(-gc, n + gc, dtype=np.float64)
        return o + i * h + 0.5 * h, np.full(n + 2 * gc, h, dtype=np.float64)
    x, hx = axis(nx, origin[0])
    y, hy = axis(ny, origin[1])
    z, hz = axis(nz, origin[2])
    return Grid(nx + 2 * gc, ny + 2 * gc, nz + 2 * gc, gc, x, y, z, hx, hy, hz)


def stretched_grid(nx, ny, nz, h, ratio=1.02, gc=GC):
    """Geometrically stretched widths along y and z (for non-uniform metric tests)."""
    def axis(n, stretch):
        w = h * stretch ** np.abs(np.arange(-gc, n + gc) - (n // 2))
        c = np.cumsum(w) - 0.5 * w
        c = c - c[gc] + 0.5 * w[gc]
        return c.astype(np.float64), w.astype(np.float64)
    x, hx = axis(nx, 1.0)
    y, hy = axis(ny, ratio)
    z, hz = axis(nz, ratio)
    return Grid(nx + 2 * gc, ny + 2 * gc, nz + 2 * gc, gc, x, y, z, hx, hy, hz)


# ---------------------------------------------------------------- turbine
def polar_table():
    """Synthetic polars on -30..30 deg every 0.5 deg: Cl = 2 pi clip(alpha, +-12 deg), Cd = 0.01 + 0.05 alpha^2."""
    attack = np.arange(-30.0, 30.0 + 0.25, 0.5)
    a = np.deg2rad(attack)
    cl = 2.0 * np.pi * np.clip(a, -np.deg2rad(12.0), np.deg2rad(12.0))
    cd = 0.01 + 0.05 * a * a
    return attack, cl, cd


def blade_stations():
    """Two stations, chord/R and twist linear from the root (r/R 0.1) to the tip
    (values of app/nedo/turbineProperties.json at r/R 0.1 and 1.0)."""
    attack, cl, cd = polar_table()
    return {
        "r": np.array([0.1, 1.0]),
        "chord": np.array([0.0771222, 0.02287395]),
        "twist": np.array([12.32334, -1.282757]),
        "cl": np.stack([cl, cl]),
        "cd": np.stack([cd, cd]),
        "attack": attack,
    }


def build_aps_py(st, apcount, n_ap_per_blade, radius, hub_radius):
    """numpy restatement of BladeHandler::buildAP (src/alm/bladeHandler.h:46-104)."""
    dr = (radius - hub_radius) / n_ap_per_blade
    r_st = st["r"]
    ns, na = st["cl"].shape
    out = {"r": np.zeros(apcount), "chord": np.zeros(apcount), "twist": np.zeros(apcount),
           "cl": np.zeros(apcount * na), "cd": np.zeros(apcount * na)}
    for ap in range(apcount):
        apr = (ap % n_ap_per_blade + 0.5) * dr + hub_radius
        if apr < r_st[0]:
            lo, w, mode = 0, 0.0, 0
        elif apr >= r_st[-1]:
            lo, w, mode = ns - 1, 0.0, 1
        else:
            for i in range(ns - 1):
                if r_st[i] <= apr < r_st[i + 1]:
                    lo, w = i, (apr - r_st[i]) / (r_st[i + 1] - r_st[i])
                    break
            mode = 2

        def itp(v):
            if mode == 0:
                return v[0]
            if mode == 1:
                return v[ns - 1]
            return (1.0 - w) * v[lo] + w * v[lo + 1]
        out["r"][ap] = apr
        out["chord"][ap] = itp(st["chord"])
        out["twist"][ap] = itp(st["twist"])
        clv, cdv = itp(st["cl"]), itp(st["cd"])
        for a in range(na):
            out["cl"][ap + a * apcount] = clv[a]
            out["cd"][ap + a * apcount] = cdv[a]
    return out


@dataclass
class AlmSetup:
    n_turbine: int
    n_blade: int
    n_ap_per_blade: int
    radius: float
    hub_radius: float
    euler_eps: float
    base: np.ndarray          # (n_turbine, 3)
    hub: np.ndarray           # (n_turbine, 3)
    tip_rate: np.ndarray
    motion: np.ndarray        # (n_turbine, 3): amplitude [rad], angular frequency, phase [rad]
    angle_type: np.ndarray    # int
    stations: dict
    aps: dict
    pitch: float = 0.0

    @property
    def apcount(self):
        return self.n_turbine * self.n_blade * self.n_ap_per_blade

    @property
    def n_attack(self):
        return len(self.stations["attack"])

    def arrays(self):
        return {
            "base": np.ascontiguousarray(self.base, dtype=np.float64).ravel(),
            "hub": np.ascontiguousarray(self.hub, dtype=np.float64).ravel(),
            "tip_rate": np.ascontiguousarray(self.tip_rate, dtype=np.float64),
            "motion": np.ascontiguousarray(self.motion, dtype=np.float64).ravel(),
            "angle_type": np.ascontiguousarray(self.angle_type, dtype=np.int32),
            "ap_r": np.ascontiguousarray(self.aps["r"]), "ap_chord": np.ascontiguousarray(self.aps["chord"]),
            "ap_twist": np.ascontiguousarray(self.aps["twist"]),
            "attack": np.ascontiguousarray(self.stations["attack"], dtype=np.float64),
            "cl": np.ascontiguousarray(self.aps["cl"]), "cd": np.ascontiguousarray(self.aps["cd"]),
        }


def make_rotor(hub_xyz, h, tsr=7.0, n_ap_per_blade=32, eps_cells=2.0, pitch=0.0,
               platform_pitch_deg=0.0, platform_period=10.0, tower=0.0):
    """One 3-blade rotor of radius 1 centred at hub_xyz (turbine base at hub_xyz - (0,0,tower))."""
    st = blade_stations()
    apc = 3 * n_ap_per_blade
    aps = build_aps_py(st, apc, n_ap_per_blade, 1.0, 0.0)
    base = np.array([[hub_xyz[0], hub_xyz[1], hub_xyz[2] - tower]])
    hub = np.array([[0.0, 0.0, tower]])
    if platform_pitch_deg:
        motion = np.array([[math.radians(platform_pitch_deg), 2 * math.pi / platform_period, 0.0]])
        atype = np.array([2], dtype=np.int32)
    else:
        motion = np.zeros((1, 3))
        atype = np.array([0], dtype=np.int32)
    return AlmSetup(1, 3, n_ap_per_blade, 1.0, 0.0, eps_cells * h, base, hub, np.array([tsr]), motion, atype,
                    st, aps, pitch)


@dataclass
class RmcpSetup:
    """The reference's RMCP rotor model (src/rmcp/turbineHandler.h, bladeHandler.h):
    turbines of a fixed orientation whose rotating blades paint the cells they
    cover.  angle_deg: one Euler angle per turbine in degrees (the reference's
    JSON unit), angle_type 0 none / 1 roll / 2 pitch / 3 yaw."""
    n_turbine: int
    n_blade: int
    radius: float
    hub_radius: float
    width: float
    thick: float
    base: np.ndarray          # (n_turbine, 3)
    hub: np.ndarray           # (n_turbine, 3): (-overhang, 0, tower)
    angle_deg: np.ndarray     # (n_turbine, 3)
    angle_type: np.ndarray
    tip_rate: np.ndarray
    stations: dict

    def arrays(self):
        st = self.stations
        return {
            "base": np.ascontiguousarray(self.base, dtype=np.float64).ravel(),
            "hub": np.ascontiguousarray(self.hub, dtype=np.float64).ravel(),
            # deg2rad as the reference converts its JSON angles (src/falmath.h:51-53)
            "angle": np.ascontiguousarray([a * math.pi / 180.0 for a in np.asarray(self.angle_deg, dtype=np.float64).ravel()]),
            "angle_type": np.ascontiguousarray(self.angle_type, dtype=np.int32),
            "tip_rate": np.ascontiguousarray(self.tip_rate, dtype=np.float64),
            "st_r": np.ascontiguousarray(st["r"], dtype=np.float64),
            "st_chord": np.ascontiguousarray(st["chord"], dtype=np.float64),
            "st_twist": np.ascontiguousarray(st["twist"], dtype=np.float64),
            "attack": np.ascontiguousarray(st["attack"], dtype=np.float64),
            "cl": np.ascontiguousarray(st["cl"], dtype=np.float64).ravel(),
            "cd": np.ascontiguousarray(st["cd"], dtype=np.float64).ravel(),
        }


def make_rmcp(hub_xyz, tsr=7.0, width=0.1, thick=0.1, yaw_deg=0.0, tower=0.0):
    """One 3-blade RMCP rotor of radius 1 centred at hub_xyz, with the reference's
    blade strip width and thickness (BLADE_WIDTH, BLADE_THICK: 0.1), the blade
    stations of blade_stations() and an optional yaw of the whole turbine"""
    base = np.array([[hub_xyz[0], hub_xyz[1], hub_xyz[2] - tower]])
    hub = np.array([[0.0, 0.0, tower]])
    ang = np.array([[0.0, 0.0, yaw_deg]])
    atype = np.array([3 if yaw_deg else 0], dtype=np.int32)
    return RmcpSetup(1, 3, 1.0, 0.0, width, thick, base, hub, ang, atype, np.array([tsr]), blade_stations())


# ---------------------------------------------------------------- inflow
def inflow_box(ny, nz, intensity, nb=128, corr=8, seed=INFLOW_SEED):
    """Periodic 3 x nb x ny x nz perturbation box: i.i.d. N(0,1) from Philox(seed),
    box-filtered over `corr` cells per axis (periodic), rescaled to std `intensity`."""
    from scipy.ndimage import uniform_filter1d
    rng = np.random.Generator(np.random.Philox(seed))
    box = rng.standard_normal((3, nb, nz, ny))           # [d][x][k][j]
    for ax in (1, 2, 3):
        box = uniform_filter1d(box, corr, axis=ax, mode="wrap")
    for d in range(3):
        box[d] *= intensity / box[d].std()
    # layout of falm_bc_set_inflow: component, x plane, then j fastest, then k
    return np.ascontiguousarray(box)


# ---------------------------------------------------------------- cases
@dataclass
class Case:
    name: str
    grid: Grid
    bc: int                     # 0 channel, 1 cavity
    Re: float
    dt: float
    tol: float
    maxit: int = 1000
    Cs: float = 0.1
    adv: str = "Upwind3"
    sgs: str = "Smagorinsky"
    pc: str = "SOR"
    pc_maxit: int = 2
    pc_relax: float = 1.2
    u_inlet: float = 1.0
    alm: AlmSetup = None
    rmcp: RmcpSetup = None
    intensity: float = 0.0
    steps: int = 1
    inflow: np.ndarray = field(default=None, repr=False)

    def with_inflow(self, nb=128):
        if self.intensity > 0 and self.inflow is None:
            nx, ny, nz = self.grid.interior
            self.inflow = inflow_box(ny, nz, self.intensity, nb=nb)
        return self


def cavity(n=64):
    g = uniform_grid(n, n, n, 1.0 / n)
    return Case("cavity", g, 1, Re=1000.0, dt=1e-3, tol=1e-8, u_inlet=0.0, steps=100)


def channel(nx=256, ny=128, nz=128, cells_per_radius=20, tsr=7.0, intensity=0.05, tol=1e-8, steps=2000,
            name="channel", n_ap_per_blade=32, hub=None):
    h = 1.0 / cells_per_radius
    g = uniform_grid(nx, ny, nz, h)
    hub = hub or (3.2, 0.5 * ny * h, 0.5 * nz * h)
    rotor = make_rotor(hub, h, tsr=tsr, n_ap_per_blade=n_ap_per_blade)
    return Case(name, g, 0, Re=1e4, dt=0.3 * h, tol=tol, alm=rotor, intensity=intensity, steps=steps)


def channel_large():
    return channel(512, 256, 256, tol=1e-6, steps=5000, name="channel_large")


def channel_half():
    """512 x 256 x 128: the x/y shape of channel_large with half the planes (profiling case)"""
    return channel(512, 256, 128, tol=1e-6, steps=5000, name="channel_half")


def adjoint_case():
    return channel(128, 64, 64, cells_per_radius=10, steps=200, name="adjoint")


def floating(intensity=0.08):
    h = 1.0 / 24
    nx, ny, nz = 1024, 256, 256
    g = uniform_grid(nx, ny, nz, h)
    rotor = make_rotor((5.0, 0.5 * ny * h, 0.5 * nz * h), h, tsr=9.0, pitch=3.0, platform_pitch_deg=3.0,
                       platform_period=10.0, tower=3.0)
    return Case("floating", g, 0, Re=1e4, dt=0.3 * h, tol=1e-6, alm=rotor, intensity=intensity, steps=3000)


def small_channel(nx=40, ny=24, nz=24, cells_per_radius=6, intensity=0.05, tol=1e-10, n_ap_per_blade=8):
    """A small channel + rotor for parity tests (the rotor fits inside the domain)."""
    h = 1.0 / cells_per_radius
    hub = (0.5 * nx * h * 0.6, 0.5 * ny * h, 0.5 * nz * h)
    c = channel(nx, ny, nz, cells_per_radius=cells_per_radius, intensity=intensity, tol=tol, steps=10,
                name="small_channel", n_ap_per_blade=n_ap_per_blade, hub=hub)
    return c


def initial_state(case):
    """Start fields as the drivers do: u = (u_inlet, 0, 0) everywhere (app/nedo/main.cpp:124-130),
    zero elsewhere; uu and nut are then derived with UtoUU and SGS."""
    n = case.grid.n
    u = np.zeros(3 * n)
    u[:n] = case.u_inlet
    return {"u": u, "uu": np.zeros(3 * n), "p": np.zeros(n), "nut": np.zeros(n), "ff": np.zeros(3 * n)}
