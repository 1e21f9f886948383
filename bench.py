#!/usr/bin/env python
"""Throughput of the FALM LES step on B200: Mcell/s (and steps/s).

Default workload: the 512x256x256 channel with one actuator-line rotor
(33.5 M interior cells, h = 1/20, TSR 7, uniform inflow U = 1, CFL 0.3) with
the Poisson tolerance at which ||div u|| stays below 1e-6 (1e-8; the case's
own 1e-6 leaves it near 2e-6), in mixed precision (FP32 storage, FP64
reductions).  Beside it: the FP64 step on the same workload (mixed/FP64),
the same grid with seeded 5% inflow turbulence in both precisions, the case
tolerance 1e-6, the field errors of mixed against FP64 after 10 steps, the
CPU oracle on a slice, and the adjoint/forward cost ratio.  One JSON line on
rank 0.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own CUDA step (built from its sources
into oracle/_ref) on the same workload (same grid, rotor, uniform inflow and
tolerance) in FP64, its only precision; if that build is absent it times the
CPU oracle.  Multi-GPU (torchrun): every rank runs its own replica of the case
(weak scaling); the time is the maximum over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "step/s & Mcell/s on 1 B200: mixed vs FP64 at div<=1e-6; adjoint/forward ratio"
UNIT = "Mcell/s"
RESTART = 100   # steps after which a timed phase returns to its starting state
DIV_TOL = 1e-8  # Poisson tolerance at which the case's ||div u|| stays below 1e-6
ADJ_TOL_FLOATING = 1e-3   # relative residual of the floating case's transposed Poisson solves


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)   # about 0.85 s of timed steps: several clock samples
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default="channel_large")
    ap.add_argument("--slabs", action="store_true",
                    help="with N ranks: one grid of N z-stacked copies of the case's planes, one slab per GPU, halos and "
                         "reductions over NCCL (weak scaling), instead of N independent replicas")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward cost ratio")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the secondary runs (seeded inflow, the case tolerance 1e-6, field errors after 10 steps)")
    ap.add_argument("--tol", type=float, default=DIV_TOL,
                    help="Poisson tolerance (default 1e-8: the case's ||div u|| stays below 1e-6)")
    ap.add_argument("--intensity", type=float, default=0.0,
                    help="inflow turbulence intensity of the timed workload (default 0: uniform inflow, as the reference)")
    ap.add_argument("--power-run", type=int, default=0, metavar="STEPS",
                    help="instead of the benchmark: time-averaged rotor power and thrust over STEPS steps, "
                         "mixed against FP64, at --power-cfl")
    ap.add_argument("--power-cfl", type=float, default=0.05)
    ap.add_argument("--configs", action="store_true",
                    help="instead of the benchmark: the step on the reference's cavity 64^3, channel "
                         "256x128x128 and 512x256x256 and floating-turbine 1024x256x256 configurations, "
                         "timed for the B200 step, the reference's CUDA step and the CPU oracle")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed plumbing
def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """the maximum of x over the ranks (nccl on the GPUs, gloo on the host)"""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, cells, steps, ms_max):
    """whole-job Mcell/s of `world` independent replicas, timed by the slowest rank"""
    return world * cells * steps / (ms_max / 1e3) / 1e6


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, its maximum, power and the throttle reasons of this process's GPU,
    sampled every 20 ms through NVML during the timed region (nvidia-smi every
    100 ms where NVML is not available).  stop() keeps sampling, for at most one
    second, until at least 3 samples were taken, so that even a short timed
    region carries a clock record."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []          # (sm_mhz, sm_max_mhz, power_w, reason bits)
        self.proc = None
        self.nvml = None
        self.stop_flag = False
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.idx)
        uuid = str(getattr(props, "uuid", "") or "")
        if uuid:
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                pass
        bus = getattr(props, "pci_bus_id", None)
        if bus is not None:
            dom = getattr(props, "pci_domain_id", 0)
            dev = getattr(props, "pci_device_id", 0)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(f"{dom:08x}:{bus:02x}:{dev:02x}.0")
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.idx)

    def _nvml_loop(self, nv, h):
        while not self.stop_flag:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), pw, int(rs)))
            except Exception:
                pass
            time.sleep(0.02)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.source = "nvml, 20 ms"
            self.thread.start()
            return self
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._smi_read, daemon=True)
            self.source = "nvidia-smi, 100 ms"
            self.thread.start()
            # the first line comes at start-up: wait for it, then keep only the
            # samples taken from here on
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 5.0:
                time.sleep(0.01)
            self.rows.clear()
        except Exception:
            self.proc = None
        return self

    def _smi_read(self):
        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                bits = 0
                for k, (_, b) in enumerate(self.REASONS):
                    if parts[5 + k].lower().startswith("active"):
                        bits |= b
                self.rows.append((num(parts[1]), num(parts[2]), num(parts[3]), bits))

    def stop(self):
        t0 = time.perf_counter()
        while self.source and len(self.rows) < 3 and time.perf_counter() - t0 < 1.0:
            time.sleep(0.01)
        self.stop_flag = True
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        rows = list(self.rows)
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(rows), "source": self.source}
        if not rows:
            return out
        sm = [r[0] for r in rows if r[0]]
        mx = [r[1] for r in rows if r[1]]
        pw = [r[2] for r in rows if r[2]]
        out["sm_mhz"] = statistics.median(sm) if sm else None
        out["sm_max_mhz"] = max(mx) if mx else None
        out["reasons"] = sorted({name for r in rows for name, bit in self.REASONS if r[3] & bit})
        out["power_w_max"] = max(pw) if pw else None
        return out


def it_summary(its):
    """BiCGStab iterations per step: the list for a few steps, else min/mean/max"""
    if len(its) <= 20:
        return its
    return {"min": min(its), "mean": sum(its) / len(its), "max": max(its), "steps": len(its)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- algorithmic bytes
def step_bytes(S, n, it, m=2):
    """bytes per step: S*N*[44 + it*(28 + 6m)] (4 B/value mixed, 8 B FP64); the ALM
    support term 3*S*N_box is negligible against N and left out"""
    return S * n * (44 + it * (28 + 6 * m))


# values moved per interior cell by one launch of each kernel class (reads + writes,
# each operand once): used for the per-kernel achieved bandwidth
KERNEL_VALUES = {
    "pseudo_u": 10,     # u(3) uu(3) nut(1) in, ua(3) out (ALM force evaluated in-kernel)
    "utouu_rhs": 10,    # ua(3) p(1) in, uu(3) rhs(1) rr(1) pp(1) out (the solve's first residual fused in)
    "res": 2,           # the mixed-precision outer check: x b in (a pass residual after a failed check: 4)
    "bicg_p": 5,        # r p q in, p pp out (from a pass's second iteration on)
    "sor": 3,           # x b in, x out (three red-black half sweeps per launch, one HBM pass)
    "mv_dot1": 3,       # pp rr in, q out
    "bicg_s": 4,        # r q in, s ss out
    "mv_dot2": 3,       # ss s in, t out
    "bicg_xr": 8,       # x pp ss s t rr in, x r out
    "project": 13,      # ua(3) uu(3) p in, u(3) uu(3) out
    "sgs_div": 7,       # u(3) uu(3) in, nut out
}


def traffic_for(kernel):
    """dram bytes per launch from the committed ncu summary, if one exists"""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


# ---------------------------------------------------------------- workload
def bench_case(args, intensity=None, tol=None):
    """The benchmark's case: the 512x256x256 channel with the rotor (the case of
    --case) at Poisson tolerance `tol` (default --tol) and inflow turbulence
    `intensity` (default: uniform inflow, which both arms run)."""
    from falm_b200 import cases
    c = getattr(cases, args.case)()
    c.tol = args.tol if tol is None else tol
    c.intensity = args.intensity if intensity is None else intensity
    c.inflow = None
    return c.with_inflow()


def workload_config(args, case):
    """the configuration dict both arms print (identical for the same arguments)"""
    g = case.grid.interior
    infl = "uniform inflow U = 1" if not case.intensity else f"seeded {case.intensity:.0%} inflow (Philox seed 20261203)"
    return {"workload": f"{case.name} {g[0]}x{g[1]}x{g[2]} channel + 3-blade ALM rotor (R = 20 cells, TSR 7, 96 APs), "
                        f"{infl}, Re 1e4, CFL 0.3, PBiCGStab + red-black SOR x{case.pc_maxit} (omega {case.pc_relax}), "
                        f"tol {case.tol:g} (||div u|| <= 1e-6)",
            "cells": case.grid.n_interior, "tol": case.tol, "inflow_intensity": case.intensity,
            "l2": "inputs larger than L2 (one FP32 field is 140 MB, one FP64 field 280 MB; L2 126 MB)"}


# ---------------------------------------------------------------- our arm
def run_ours(args, rank, world, local):
    import torch
    from falm_b200.driver import Simulation
    case = bench_case(args)
    n = case.grid.n_interior
    out = {}

    def timed(sim, K, e2e=False):
        # Every phase starts from the state kept after the warm-up, and the run
        # goes back to it every RESTART steps (device copies of the fields,
        # inside the timed region): at CFL 0.3 the explicit-Euler step with the
        # Upwind3 scheme amplifies mid-wavenumber modes, and the flow leaves the
        # stable range after about 240 (seeded inflow) or 450 (uniform) steps.
        ctx = sim.ctx
        sim.restore()
        planes = None
        if e2e:
            planes = [torch.from_numpy(sim.inlet_plane(sim.it + 1 + q)).pin_memory() for q in range(min(K, RESTART))]
        torch.cuda.synchronize()
        barrier(world)
        l0 = ctx.launches()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []
        wall0 = time.perf_counter()
        ev0.record()
        for q in range(K):
            if q and q % RESTART == 0:
                sim.restore()
            if e2e:
                ctx.set_inlet_plane(planes[q % RESTART])
            stats.append(sim.step())
        ev1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        ms = ev0.elapsed_time(ev1)
        barrier(world)
        return ms, stats, ctx.launches() - l0, wall

    def arm(c, prec, K):
        """W warm-up steps, then K timed steps; returns the summary and the stats"""
        sim = Simulation(c, prec)
        for _ in range(args.warmup):
            sim.step()
        sim.snapshot()
        ms, st, _, _ = timed(sim, K)
        ms = max_over_ranks(ms, world)
        its = [x["it"] for x in st]
        sb = step_bytes(4 if prec == "mixed" else 8, n, sum(its) / len(its))
        res = {"value": replica_rate(world, n, K, ms), "ms_per_step": ms / K, "steps_per_s": 1e3 * K / ms,
               "its": it_summary(its), "outer_max": max(x["outer"] for x in st),
               "divnorm_max": max(x["divnorm"] for x in st), "step_roofline_frac": sb / (ms / K / 1e3) / 1e9 / peak}
        sim.close()
        del sim
        torch.cuda.empty_cache()
        return res

    peak, peak_kind = peaks()
    sim = Simulation(case, args.precision)
    for _ in range(args.warmup):
        sim.step()
    sim.snapshot()
    clocks = ClockSampler(local).start()
    ms, stats, launches, wall = timed(sim, args.steps)
    clk = clocks.stop()
    # per-kernel device times (CUDA events around every launch) from the same
    # number of further steps: events between launches would also break the
    # overlap of consecutive kernels that the timed steps use
    sim.ctx.profile(True)
    sim.ctx.profile_read(reset=True)
    timed(sim, args.steps)
    prof = sim.ctx.profile_read(reset=True)
    sim.ctx.profile(False)
    ms_max = max_over_ranks(ms, world)
    S = 4 if args.precision == "mixed" else 8
    its = [s["it"] for s in stats]
    mean_it = sum(its) / len(its)
    value = replica_rate(world, n, args.steps, ms_max)
    # dominant kernel class by device time
    cls = max((k for k in prof if k in KERNEL_VALUES), key=lambda k: prof[k][0])
    tms, tn = prof[cls]
    avg_ms = tms / max(tn, 1)
    alg_bytes = KERNEL_VALUES[cls] * S * n
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    step_b = step_bytes(S, n, mean_it)
    divmax = max(s["divnorm"] for s in stats)
    out.update({
        "value": value, "ms_per_step": ms_max / args.steps, "steps_per_s": 1e3 * args.steps / ms_max,
        "launches": launches, "its": it_summary(its), "divnorm_max": divmax, "div_ok": divmax <= 1e-6,
        "err_max": max(s["err"] for s in stats), "clocks": clk,
        "roofline": {"bound": "hbm", "kernel": cls, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic_for(cls), "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms},
        "step_roofline": {"bytes_per_step": step_b, "achieved": step_b / (ms_max / args.steps / 1e3) / 1e9,
                          "frac": step_b / (ms_max / args.steps / 1e3) / 1e9 / peak, "it": mean_it, "m": case.pc_maxit},
        "profile": {k: {"ms": v[0], "launches": v[1]} for k, v in prof.items() if v[1]},
        "wall_s": wall,
    })
    if not args.no_e2e:
        ms_e, stats_e, _, wall_e = timed(sim, args.steps, e2e=True)
        ms_e = max_over_ranks(ms_e, world)
        ny, nz = case.grid.interior[1], case.grid.interior[2]
        out["e2e"] = {"value": replica_rate(world, n, args.steps, ms_e), "unit": UNIT,
                      "h2d_bytes_per_step": 3 * ny * nz * 8,
                      "d2h_bytes_per_step": 8 * 8 + 2 * 8 * 8,
                      "ms_per_step": ms_e / args.steps,
                      "note": "per step: the inlet velocity plane (3 x nz x ny FP64) copied H2D from pinned host memory, "
                              "falm_step through the C ABI, step statistics (it, err, div norm, torque, thrust) read "
                              "back to the host"}
    sim.close()
    del sim
    torch.cuda.empty_cache()
    if args.precision == "mixed" and not args.no_fp64:
        out["fp64"] = arm(case, "fp64", args.steps)
        out["fp64"]["note"] = ("our FP64 step on the same workload; the reference arm (--impl reference) prints "
                               "the reference's FP64 step on it")
        out["mixed_over_fp64"] = out["fp64"]["ms_per_step"] / out["ms_per_step"]
    if args.precision == "mixed" and not args.no_extra:
        K = min(args.steps, RESTART)
        # the benchmark configuration's own physics: seeded 5% inflow turbulence
        seeded = bench_case(args, intensity=0.05)
        sd = {"config": workload_config(args, seeded)["workload"], "steps": K,
              "mixed": arm(seeded, "mixed", K), "fp64": arm(seeded, "fp64", K)}
        sd["mixed_over_fp64"] = sd["fp64"]["ms_per_step"] / sd["mixed"]["ms_per_step"]
        out["seeded_inflow"] = sd
        # the case's own Poisson tolerance, 1e-6, which leaves ||div u|| near 2e-6 with the seeded inflow
        loose = bench_case(args, tol=1e-6)
        out["tol_1e-6"] = {"note": "secondary: the case's tolerance 1e-6 does not guarantee ||div u|| <= 1e-6 "
                                   "(1.95e-6 with the seeded 5% inflow); see divnorm_max",
                           "mixed": arm(loose, "mixed", K)}
        out["fields_10_steps"] = {"uniform_inflow": field_errors(case), "seeded_inflow": field_errors(seeded)}
    return case, out


def field_errors(case, steps=10):
    """mixed precision against the FP64 step after `steps` steps from the same
    initial state: relative L2 of u, uu, p, nut over the interior, and the
    relative differences of rotor power and thrust at the last step (the FP64
    step matches the CPU oracle and the reference's step at 1e-10 on the
    parity grids)"""
    import torch
    from falm_b200.driver import Simulation
    res, keep = {}, {}
    for prec in ("fp64", "mixed"):
        sim = Simulation(case, prec)
        for _ in range(steps):
            st = sim.step()
        g = case.grid
        gc = g.gc
        keep[prec] = ({k: getattr(sim, k).view(-1, g.sz, g.sy, g.sx)[:, gc:-gc, gc:-gc, gc:-gc].double().clone()
                       for k in ("u", "p", "nut")}, st)
        uu = sim.uu.view(3, g.sz, g.sy, g.sx)[:, gc - 1:-gc, gc - 1:-gc, gc - 1:-gc].double().clone()
        keep[prec][0]["uu"] = uu
        sim.close()
        del sim
        torch.cuda.empty_cache()
    a, sa = keep["mixed"]
    b, sb = keep["fp64"]
    for k in ("u", "uu", "p", "nut"):
        res[k] = float(torch.linalg.vector_norm(a[k] - b[k]) / torch.linalg.vector_norm(b[k]))
    res["power"] = abs(sa["torque"][0] - sb["torque"][0]) / abs(sb["torque"][0])
    res["thrust"] = abs(sa["thrust"][0] - sb["thrust"][0]) / abs(sb["thrust"][0])
    res["steps"] = steps
    del keep
    torch.cuda.empty_cache()
    return res


def run_configs(args):
    """The step on the reference's configurations, each timed three ways on this
    box: the B200 step (FP64 and mixed; fields in HBM, CUDA events on the
    stream), the reference's own CUDA step (FP64, uniform inflow, wall clock
    between synchronisations) and the CPU oracle (FP64, all host threads, a
    bounded number of steps after one untimed step). Every timed run starts 3
    steps in and returns to that state every RESTART steps."""
    import tempfile
    import numpy as np
    import torch
    from falm_b200 import cases
    from falm_b200.driver import Simulation
    from oracle.oracle import CaseStruct, Oracle, RefStep, build
    # (name, case, timed steps, CPU oracle steps, the reference's input: the
    # channels with uniform inflow, as the reference has no seeded inflow)
    defs = [("C1 cavity 64^3 (Re 1000, dt 1e-3, tol 1e-8)", cases.cavity(64), 100, 100, None),
            ("C2 channel 256x128x128 + rotor (5% inflow, CFL 0.3, tol 1e-8)", cases.channel(256, 128, 128).with_inflow(), 100, 3,
             cases.channel(256, 128, 128, intensity=0.0)),
            ("C3 channel 512x256x256 + rotor (5% inflow, CFL 0.3, tol 1e-6)", cases.channel_large().with_inflow(), 100, 0,
             cases.channel(512, 256, 256, intensity=0.0, tol=1e-6, name="channel_large_uniform")),
            ("C5 floating turbine 1024x256x256, forward step (8% inflow, platform pitch 3 deg, TSR 9, tol 1e-6)",
             cases.floating().with_inflow(), 100, 0, cases.floating(intensity=0.0))]
    ref_ok = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libfalmref.so"))
    build()
    lines = []
    for name, case, K, kcpu, uniform in defs:
        n = case.grid.n_interior
        row = {"config": name, "cells": n, "steps": K, "unit": UNIT}
        runs = [("fp64", case), ("mixed", case)]
        if uniform is not None:
            runs += [("fp64_uniform_inflow", uniform), ("mixed_uniform_inflow", uniform)]
        for key, c in runs:
            prec = "fp64" if key.startswith("fp64") else "mixed"
            sim = Simulation(c, prec)
            for _ in range(3):
                sim.step()
            sim.snapshot()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            its = []
            e0.record()
            for q in range(K):
                if q and q % RESTART == 0:
                    sim.restore()
                its.append(sim.step()["it"])
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / K
            row[key] = {"value": n / ms / 1e3, "ms_per_step": ms, "its_mean": sum(its) / K}
            sim.close()
            del sim
            torch.cuda.empty_cache()
        row["mixed_over_fp64"] = row["fp64"]["ms_per_step"] / row["mixed"]["ms_per_step"]
        if ref_ok:
            ref = RefStep(CaseStruct(uniform or case, use_inflow=False), tempfile.mkdtemp(prefix="falmref_"))
            st = cases.initial_state(uniform or case)
            ref.set("U", st["u"])
            ref.op("UTOUU")
            ref.op("SGS")
            it = 0
            for _ in range(3):
                it += 1
                ref.step(it * case.dt)
            snap = {k: ref.get(k) for k in ("U", "UU", "P", "NUT")}
            it0, el, its = it, 0.0, []
            for q0 in range(0, K, RESTART):
                if q0:
                    for k, v in snap.items():
                        ref.set(k, v)
                    it = it0
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                for _ in range(min(RESTART, K - q0)):
                    it += 1
                    its.append(ref.step(it * case.dt)["it"])
                torch.cuda.synchronize()
                el += time.perf_counter() - t0
            ref.close()
            ms = 1e3 * el / K
            row["reference_gpu"] = {"value": n / ms / 1e3, "ms_per_step": ms, "its_mean": sum(its) / K}
            mine = row["mixed_uniform_inflow" if uniform is not None else "mixed"]
            row["mixed_over_reference"] = ms / mine["ms_per_step"]
        if kcpu:
            O = Oracle()
            cs = CaseStruct(case)
            m = O.setup(cs)
            st = cases.initial_state(case)
            O.init_state(cs, m, st)
            O.step(cs, st, m, case.dt)
            t0 = time.perf_counter()
            for q in range(kcpu):
                O.step(cs, st, m, (q + 2) * case.dt)
            el = time.perf_counter() - t0
            row["cpu_oracle"] = {"value": n * kcpu / el / 1e6, "ms_per_step": 1e3 * el / kcpu, "cores": O.threads(),
                                 "steps": kcpu}
        lines.append(row)
        print(json.dumps(row), flush=True)
    return lines


def power_run(args):
    """Time-averaged rotor power and thrust over a long run, mixed precision
    against FP64 (the FP64 step matches the CPU oracle step for step), on the
    bench case at a Courant number where the explicit step is stable."""
    from falm_b200 import cases
    from falm_b200.driver import Simulation
    import numpy as np
    import torch
    res = {}
    for prec in ("fp64", "mixed"):
        c = getattr(cases, args.case)().with_inflow()
        c.dt = c.dt * args.power_cfl / 0.3
        sim = Simulation(c, prec)
        omega = float(c.alm.tip_rate[0])
        P, T, its, div = [], [], [], 0.0
        t0 = time.perf_counter()
        for _ in range(args.power_run):
            st = sim.step()
            P.append(st["torque"][0] * omega)
            T.append(st["thrust"][0])
            its.append(st["it"])
            div = max(div, st["divnorm"])
        el = time.perf_counter() - t0
        P, T = np.array(P), np.array(T)
        h = len(P) // 2
        res[prec] = {"power_mean": float(P.mean()), "thrust_mean": float(T.mean()),
                     "power_mean_2nd_half": float(P[h:].mean()), "thrust_mean_2nd_half": float(T[h:].mean()),
                     "its_mean": float(np.mean(its)), "divnorm_max": div, "umax_end": float(sim.u.abs().max()),
                     "wall_s": el}
        sim.close()
        del sim
        torch.cuda.empty_cache()
    a, b = res["mixed"], res["fp64"]
    rel = {k: abs(a[k] - b[k]) / abs(b[k]) for k in ("power_mean", "thrust_mean", "power_mean_2nd_half", "thrust_mean_2nd_half")}
    return {"power_run": {"case": args.case, "steps": args.power_run, "cfl": args.power_cfl, "tol": getattr(cases, args.case)().tol,
                          "fp64": b, "mixed": a, "rel_diff": rel}}


def cpu_baseline(args, steps=7, warm=2):
    """the CPU oracle (OpenMP, all host threads) on a bounded sample of the
    workload: the median time of `steps` steady-state steps after `warm` untimed
    ones, on a 256x256x128 slice of the case (same h, rotor, tolerance and
    inflow), about 10-20 s of CPU work"""
    from oracle.oracle import CaseStruct, Oracle, build
    from falm_b200 import cases
    build()
    O = Oracle()
    big = bench_case(args)
    nx, ny, nz = big.grid.interior
    sx, sy, sz = max(nx // 2, 32), max(ny, 32), max(nz // 2, 32)
    h = float(big.grid.hx[big.grid.gc])
    sample = cases.channel(sx, sy, sz, cells_per_radius=round(1 / h), intensity=big.intensity, tol=big.tol,
                           hub=(3.2, 0.5 * sy * h, 0.5 * sz * h), name="cpu_sample").with_inflow()
    cs = CaseStruct(sample)
    m = O.setup(cs)
    st = cases.initial_state(sample)
    O.init_state(cs, m, st)
    for q in range(warm):
        O.step(cs, st, m, (q + 1) * sample.dt)
    times, its = [], []
    for q in range(steps):
        t0 = time.perf_counter()
        its.append(O.step(cs, st, m, (warm + q + 1) * sample.dt)["it"])
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": sample.grid.n_interior / med / 1e6, "unit": UNIT, "cores": O.threads(), "kind": "port",
            "ms_per_step": 1e3 * med, "its": its,
            "sample": f"median of {steps} FP64 steps (after {warm} untimed) of a {sx}x{sy}x{sz} slice of the workload "
                      f"(same h, rotor, tolerance and inflow), CPU oracle on {O.threads()} threads"}


# ---------------------------------------------------------------- adjoint cost
def adjoint_ratio(steps=200, checkpoint=20):
    """cost of the mean-power gradient by the discrete adjoint (forward with
    checkpoints, recomputation, reverse sweep) over the plain forward window, on
    the 128x64x64 adjoint case (rotor radius 10 cells, 32 APs per blade), FP64"""
    import torch
    from falm_b200 import adjoint as A
    from falm_b200 import cases
    from falm_b200.driver import Simulation
    case = cases.adjoint_case().with_inflow()
    sim = Simulation(case, "fp64")
    for _ in range(10):
        sim.step()
    start = (sim.it, A._clone(sim))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fwd_its = []
    J = 0.0
    for _ in range(steps):
        s = sim.step()
        fwd_its.append(s["it"])
        J += A._power(sim, s) / steps
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    A._restore(sim, start[1])
    sim.it = start[0]
    # the default: every state kept in HBM when it fits (no recomputation); the
    # first call also allocates the state buffer, so it is timed on a second call
    kept = A.auto_checkpoint(sim, steps)
    A.mean_power_gradient(sim, steps, kept)
    A._restore(sim, start[1])
    sim.it = start[0]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J2, gp, gc, gt = A.mean_power_gradient(sim, steps, kept)
    torch.cuda.synchronize()
    t_adj = time.perf_counter() - t0
    # checkpoints every `checkpoint` steps, segments recomputed
    A._restore(sim, start[1])
    sim.it = start[0]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    A.mean_power_gradient(sim, steps, checkpoint)
    torch.cuda.synchronize()
    t_ck = time.perf_counter() - t0
    # binomial checkpointing within a memory budget of 10 states (start, end and
    # scratch included): 7 checkpoint slots
    A._restore(sim, start[1])
    sim.it = start[0]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Jb, gpb, _, _ = A.mean_power_gradient_binomial(sim, steps, snaps=7)
    torch.cuda.synchronize()
    t_bin = time.perf_counter() - t0
    # device time per kernel class of one more gradient (the adjoint's own kernels are "other")
    A._restore(sim, start[1])
    sim.it = start[0]
    sim.ctx.profile(True)
    sim.ctx.profile_read(reset=True)
    A.mean_power_gradient(sim, steps, kept)
    prof = {k: [round(v[0], 3), v[1]] for k, v in sim.ctx.profile_read(reset=True).items() if v[1]}
    sim.ctx.profile(False)
    sim.close()
    g = case.grid.interior
    return {"workload": f"{case.name} {g[0]}x{g[1]}x{g[2]} + rotor (R = 10 cells, 3x32 APs), FP64, tol {case.tol}",
            "objective": f"mean rotor power over {steps} steps",
            "states_kept": "all" if kept >= steps else f"checkpoint every {kept}",
            "forward_ms": 1e3 * t_fwd, "gradient_ms": 1e3 * t_adj, "ratio": t_adj / t_fwd,
            "ratio_checkpointed": t_ck / t_fwd, "checkpoint_every": checkpoint,
            "ratio_binomial": t_bin / t_fwd, "binomial_states": 10,
            "binomial_forward_steps": A.binomial_forward_steps(steps, 7), "dJ_dpitch_binomial": gpb,
            "J": J2, "dJ_dpitch": gp, "n_params": 1 + len(gc) + len(gt), "forward_its_mean": statistics.mean(fwd_its),
            "profile_ms_launches": prof,
            "note": "gradient_ms = forward window keeping the states + reverse sweep (transposed Poisson solves to "
                    "relative residual 1e-5); ratio_checkpointed adds the recomputation of all but the last "
                    "segment; ratio_binomial stores at most 10 states and recomputes along the binomial schedule; "
                    "wall clock, each step synchronises"}


def adjoint_floating(steps=50):
    """the gradient of the mean rotor power over the final `steps` steps of the
    1024x256x256 floating-turbine case (67 M cells, TSR 9, platform pitch 3 deg)
    by the mixed-precision adjoint (FP32 states, FP64 adjoint) with binomial
    checkpointing in a quarter of the free device memory, against the forward
    window's time"""
    import torch
    from falm_b200 import adjoint as A
    from falm_b200 import cases
    from falm_b200.driver import Simulation
    case = cases.floating().with_inflow()
    sim = Simulation(case, "mixed")
    # transposed solves to relative residual 1e-3: the forward solve at the
    # case's tolerance (1e-6 per cell) stops after about one BiCGStab iteration
    sim.ctx.adjoint_set_tol(ADJ_TOL_FLOATING)
    for _ in range(5):
        sim.step()
    start = (sim.it, A._clone(sim))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its = []
    for _ in range(steps):
        its.append(sim.step()["it"])
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    A._restore(sim, start[1])
    sim.it = start[0]
    budget = 0.25 * torch.cuda.mem_get_info(sim.u.device)[0]
    snaps = max(0, min(A.snaps_for_budget(sim, budget) - 2, steps - 1))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J, gp, gc, gt = A.mean_power_gradient_binomial(sim, steps, snaps=snaps)
    torch.cuda.synchronize()
    t_adj = time.perf_counter() - t0
    free, total = torch.cuda.mem_get_info(sim.u.device)
    sim.close()
    g = case.grid.interior
    return {"workload": f"floating {g[0]}x{g[1]}x{g[2]} + rotor (TSR 9, platform pitch 3 deg, 8% inflow), mixed precision, "
                        f"tol {case.tol}",
            "objective": f"mean rotor power over {steps} steps", "forward_ms": 1e3 * t_fwd, "gradient_ms": 1e3 * t_adj,
            "ratio": t_adj / t_fwd, "binomial_snaps": snaps, "binomial_forward_steps": A.binomial_forward_steps(steps, snaps),
            "state_mb_fp32": A.state_bytes(sim) / 2 ** 20, "device_used_gb": (total - free) / 1e9,
            "J": J, "dJ_dpitch": gp, "n_params": 1 + len(gc) + len(gt), "forward_its_mean": statistics.mean(its),
            "adjoint_solve_rel_tol": ADJ_TOL_FLOATING,
            "note": "FP32 forward steps, states and checkpoints; FP64 adjoint fields, gradient and transposed Poisson "
                    "solves; at most binomial_snaps stored states "
                    "besides the start, the end and one scratch state; wall clock, each step synchronises"}


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank, world, local):
    """The reference's own CUDA step (oracle/_ref, compiled from its sources) on
    the same workload: same grid, rotor, uniform inflow and Poisson tolerance,
    in FP64 (its only precision).  Wall clock between device synchronisations
    around each segment of steps."""
    case = bench_case(args)
    n = case.grid.n_interior
    from oracle.oracle import REF_SO
    if not os.path.exists(REF_SO) or case.intensity:
        cb = cpu_baseline(args)
        return case, {"value": cb["value"], "ms_per_step": cb["ms_per_step"], "kind": "port", "cpu_baseline": cb,
                      "device": "cpu", "note": "the reference's build is absent (or the workload has seeded inflow, "
                                               "which the reference has no input for): the CPU oracle is timed"}
    import tempfile
    import torch
    from falm_b200 import cases
    from oracle.oracle import CaseStruct, RefStep
    cs = CaseStruct(case, use_inflow=False)
    ref = RefStep(cs, tempfile.mkdtemp(prefix="falmref_"))
    st = cases.initial_state(case)
    ref.set("U", st["u"])
    ref.op("UTOUU")
    ref.op("SGS")
    it = 0
    for _ in range(args.warmup):
        it += 1
        ref.step(it * case.dt)
    # the reference's flow also leaves the stable range of its explicit-Euler
    # step at CFL 0.3 (after about 450 steps with uniform inflow): the run goes
    # back to the state after the warm-up every RESTART steps, between timed
    # segments (host copies of its FP64 fields)
    snap = {k: ref.get(k) for k in ("U", "UU", "P", "NUT")}
    it0 = it
    torch.cuda.synchronize()
    clocks = ClockSampler(local).start()
    el = 0.0
    stats = []
    for q0 in range(0, args.steps, RESTART):
        if q0:
            for k, v in snap.items():
                ref.set(k, v)
            it = it0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(min(RESTART, args.steps - q0)):
            it += 1
            stats.append(ref.step(it * case.dt))
        torch.cuda.synchronize()
        el += time.perf_counter() - t0
    clk = clocks.stop()
    ref.close()
    return case, {"value": n * args.steps / el / 1e6, "ms_per_step": 1e3 * el / args.steps, "device": "gpu",
                  "its": it_summary([s["it"] for s in stats]), "divnorm_max": max(s["divnorm"] for s in stats),
                  "clocks": clk, "kind": "reference"}


def run_slabs_bench(args, rank, world, local):
    """The case's grid stacked `world` times along z (each rank one slab of the
    case's size: weak scaling), every rank a SlabSimulation over the NCCL
    transport; W warm-up steps, then K timed steps between barriers (CUDA
    events on each rank's stream, maximum over the ranks).  The state after the
    warm-up is restored every RESTART steps inside the timed region."""
    import ctypes
    import torch
    from falm_b200 import _lib as L
    from falm_b200 import cases
    from falm_b200 import slab as SL
    base = bench_case(args)
    nx, ny, nz = base.grid.interior
    h = float(base.grid.hx[base.grid.gc])
    case = cases.channel(nx, ny, nz * world, cells_per_radius=round(1 / h), intensity=args.intensity, tol=args.tol,
                         hub=(3.2, 0.5 * ny * h, 0.5 * nz * h), name=f"{base.name}_stacked{world}").with_inflow()
    transport = SL.nccl_transport(rank, world)
    sim = SL.SlabSimulation(case, rank, world, transport, args.precision, f"cuda:{local}")
    for _ in range(args.warmup):
        sim.step()
    snap = ({k: getattr(sim, k).clone() for k in ("u", "uu", "p", "nut")}, sim.it)
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local).start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    ev0.record()
    for q in range(args.steps):
        if q and q % RESTART == 0:
            for k, v in snap[0].items():
                getattr(sim, k).copy_(v)
            sim.it = snap[1]
        stats.append(sim.step())
    ev1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    barrier(world)
    clk = clocks.stop()
    n = case.grid.n_interior
    sim.close()
    L.load().falm_nccl_transport_destroy(ctypes.byref(transport))
    return case, {"value": n * args.steps / (ms / 1e3) / 1e6, "ms_per_step": ms / args.steps,
                  "steps_per_s": 1e3 * args.steps / ms, "its": it_summary([x["it"] for x in stats]),
                  "divnorm_max": max(x["divnorm"] for x in stats), "clocks": clk}


def main():
    args = parse()
    if args.power_run:
        print(json.dumps(power_run(args)), flush=True)
        return
    if args.configs:
        run_configs(args)
        return
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        if rank != 0:
            return
        case, r = run_reference(args, rank, 1, local)
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r.get("ms_per_step"),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "device": r["device"], "config": workload_config(args, case),
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "its": r.get("its"), "divnorm_max": r.get("divnorm_max"), "clocks": r.get("clocks"),
                "note": "the reference's own CUDA step (oracle/_ref, compiled from its sources for sm_100a; the "
                        "reference has no CPU implementation of the step), FP64, one GPU; rank 0 only"}
        if "cpu_baseline" in r:
            line["cpu_baseline"] = r["cpu_baseline"]
            line["note"] = r["note"]
        else:
            line["cpu_baseline"] = {"value": r["value"], "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": "the reference's own CUDA step (it has no CPU path), full workload"}
        print(json.dumps(line), flush=True)
        return
    if args.slabs:
        case, r = run_slabs_bench(args, rank, world, local)
        if rank == 0:
            g = case.grid.interior
            print(json.dumps({
                "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "steps_per_s": r["steps_per_s"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 storage / f64 reductions" if args.precision == "mixed" else "f64",
                "data": "synthetic" + (" (seeded Philox inflow, seed 20261203)" if case.intensity else " (uniform inflow)"),
                "config": workload_config(args, bench_case(args)), "precision": args.precision,
                "parallelism": f"z slabs x{world} (NCCL halos and reductions)",
                "slab_grid": f"{g[0]}x{g[1]}x{g[2]}", "its": r["its"], "divnorm_max": r["divnorm_max"],
                "clocks": r["clocks"]}), flush=True)
        return
    case, r = run_ours(args, rank, world, local)
    if rank != 0:
        return
    cb = None
    if world == 1 and not args.no_cpu:
        try:
            cb = cpu_baseline(args)
        except Exception as e:   # the baseline is reported, never required
            cb = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": f"failed: {e}"}
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "steps_per_s": r["steps_per_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 storage / f64 reductions" if args.precision == "mixed" else "f64",
        "data": "synthetic" + (" (seeded Philox inflow, seed 20261203)" if case.intensity else " (uniform inflow)"),
        "config": workload_config(args, case),
        "precision": args.precision,
        "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
        "restart": f"the state after the warm-up is restored every {RESTART} steps inside the timed region "
                   f"(device copies, counted in the time)",
        "clocks": r["clocks"], "gpu_launches": r["launches"], "roofline": r["roofline"],
        "step_roofline": r["step_roofline"], "its": r["its"], "divnorm_max": r["divnorm_max"], "div_ok": r["div_ok"],
        "err_max": r["err_max"], "profile": r["profile"],
    }
    for k in ("e2e", "fp64", "mixed_over_fp64", "seeded_inflow", "tol_1e-6", "fields_10_steps"):
        if k in r:
            line[k] = r[k]
    if cb:
        line["cpu_baseline"] = cb
    if world == 1 and not args.no_adjoint:
        try:
            line["adjoint"] = adjoint_ratio()
        except Exception as e:   # reported, never required
            line["adjoint"] = {"error": str(e)}
        try:
            line["adjoint_floating"] = adjoint_floating()
        except Exception as e:
            line["adjoint_floating"] = {"error": str(e)}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
