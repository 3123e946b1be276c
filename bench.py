#!/usr/bin/env python3
"""Benchmark of the OpenCFD-SC RHS + RK3 hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload tgv256_omp6_char] [--precision fp64|mixed]

One "step" is one RK3 time step (three stages) of the whole grid.  The
default workload is the Taylor-Green vortex on a 256^3 periodic box with the
characteristic flux path and OMP6, FP64 (the reference's du_inviscous_Character
+ du_viscous + OCFD_time_adv_RK3 + comput_duvwT + OCFD_bc per stage).  The
stated dt of 0.002 is above the stability limit of RK3 with these schemes at
Ma 0.1 on 256^3 (acoustic CFL 0.9 per direction; the oracle stops with the
reference's negative-temperature error after 17 steps at that CFL, and after 21
steps at dt = 0.001 for the characteristic OMP6 path); dt = 0.0005 (CFL 0.22)
is used.  The metric does not depend on dt.

The metric compares FP64 with mixed precision at a stated error: an FP64 line
(the default) carries a "mixed" object timed the same way -- FP32 flux
splitting, characteristic projection, reconstruction and viscous derivatives,
FP64 state, metrics, primitive recovery and RK3 combination -- with its speed
over FP64 and its errors against the FP64 run (kinetic energy and enstrophy
histories, relative L2 / Linf of rho, u and p) after the workload's stated
number of steps, both runs from the same initial field.

The same line carries a "served" object: a compact seeded stream of 64
mixed-size requests served with continuous batching (aggregate GPts/s, p50/p99
time to result) against the same requests solved one after another in FP64
and in mixed precision (`--serve` runs the full 256-request stream with errors
against FP64).

Multi-GPU: the path does not shard in this build (one grid per GPU); N GPUs run
N independent replicas ("replicas only", weak scaling), the time is the max
over ranks and the value is the total grid-point updates of all ranks.

--impl reference times the CPU restatement of the reference (the oracle, all
host threads via OpenMP) on the same configuration: each of its steps is one
full time step of the workload's own grid (the 512^3 isotropic turbulence,
about 80 GB on the host, is sampled on 128^3).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "opencfd-sc_b200"))

METRIC = "grid-pt RK3 updates/s FP64 vs mixed at stated L2 err; served p50/p99 latency"
UNIT = "GPts/s"

WORKLOADS = {
    # name: (grid, scheme, character, split, dt, description)
    "tgv256_omp6_char": (256, "OMP6", 1, 1, 0.0005, "Taylor-Green vortex 256^3, characteristic flux, OMP6, SW, CD6"),
    "tgv256_hybrid_char": (256, "HYBRID", 1, 1, 0.0005, "Taylor-Green vortex 256^3, characteristic flux, hybrid UD7L(CD8)/WENO7/WENO5, SW"),
    "tgv64_weno7": (64, "WENO7", 0, 1, 0.005, "Taylor-Green vortex 64^3, flux-vector form, WENO7, SW, CD6"),
    "tgv256_weno7": (256, "WENO7", 0, 1, 0.0005, "Taylor-Green vortex 256^3, flux-vector form, WENO7, SW, CD6"),
}


# Workloads with their own grid and initial field: name -> description
CASE_WORKLOADS = {
    "hit512_hybrid_llf": "Decaying isotropic turbulence 512^3, Mt 0.6, Re_lambda 100, hybrid (sensor 1) "
                         "UD7L(CD8)/WENO7/WENO5, LLF, flux-vector form, dt at CFL 0.5",
    "cylinder_weno7_char": "Mach 6 blunt cylinder 301x401x8, body-fitted grid, isothermal wall Tw 3, Re 1e5, "
                           "WENO7 characteristic, SW, dt 2e-5",
}


def make_case(workload: str, precision: str):
    """(params, coordinates or None, interior primitives) of a workload."""
    import math

    import numpy as np

    from ocfd_b200 import cases

    if workload in WORKLOADS:
        p = make_params(workload, precision)
        return p, None, cases.tgv_prims(p)
    if workload == "cylinder_weno7_char":
        p = cases.cylinder_params()
        p.precision = 1 if precision == "mixed" else 0
        return p, cases.cylinder_grid(p.nx, p.ny, p.nz), cases.cylinder_prims(p.nx, p.ny, p.nz)
    if workload == "hit512_hybrid_llf":
        from ocfd_b200.solver import Solver

        n, mt, ma = 512, 0.6, 1.0
        prims = cases.hit_prims(n, mt=mt, ma=ma)
        vmax = float(np.max(np.abs(prims[1]) + np.abs(prims[2]) + np.abs(prims[3]) + np.sqrt(prims[4]) / ma))
        dt = 0.5 * (2.0 * math.pi / n) / vmax
        # Re from the Taylor-scale Reynolds number of the same spectrum at 128^3 and Re = 1
        # (Re_lambda is proportional to Re; the statistics of the k0 = 4 spectrum are
        # resolved at both sizes)
        q = cases.hit_params(128, re=1.0, ma=ma, dt=dt)
        s = Solver(q)
        s.init_mesh(*cases.hit_coords(128))
        s.init3d(cases.hit_prims(128, mt=mt, ma=ma))
        re = 100.0 / float(s.ana_box()[1])
        s.close()
        p = cases.hit_params(n, re=re, ma=ma, dt=dt, mixed=precision == "mixed")
        return p, cases.hit_coords(n), prims
    raise ValueError(workload)


def make_params(workload: str, precision: str, n_override: int | None = None):
    from ocfd_b200 import cases
    from ocfd_b200.params import SCHEME

    n, scheme, chr_, split, dt, _ = WORKLOADS[workload]
    if n_override:
        n = n_override
    if chr_ == 1:
        p = cases.tgv_char_params(n, scheme, dt=dt)
    else:
        p = cases.tgv_params(n, scheme=SCHEME[scheme], character=chr_, split=split, dt=dt)
    p.precision = 1 if precision == "mixed" else 0
    return p


# ---------------------------------------------------------------------------------------------
# byte model (algorithmic bytes per grid point, per launch) of each kernel group
def byte_model(p, zero_mask: int = 0) -> dict:
    """Algorithmic bytes per grid point of each kernel launch.  zero_mask: the
    metric arrays the library found identically zero (their loads are skipped)."""
    r = 4 if p.precision == 1 else 8  # face fluxes / Ev / FP32 copies of prims+metrics
    s = 4 if p.precision == 1 else 8  # prims + metric rows read by the face kernels
    nz = lambda ms: sum(1 for m in ms if not (zero_mask >> m) & 1)
    nface = 5  # characteristic form: projected fluxes; flux-vector form: h(F+) + h(F-) per face
    face = {d: 5 * s + nz(range(13 + 3 * i, 16 + 3 * i)) * s + nface * r for i, d in enumerate(("x", "y", "z"))}
    # u,v,w,T + the non-zero metrics Akx..Asz and Akx1..Asz1 in (not Ajac); 12 Ev out
    visc = 4 * s + nz(list(range(3, 12)) + list(range(13, 22))) * s + 12 * r
    # tail: 3 directions of faces + 12 Ev + Ajac + fn + f (2 of 3 stages) in; f + prims out.
    # Mixed precision on an all-periodic grid (BC_None, fused): stages 1-2 write only T of
    # the FP64 primitives; FP32 copies of d and u,v,w,T (20 bytes) every stage.
    lean = p.precision == 1 and all(p.iperiodic[d] for d in range(3)) and p.if_mass_force != 1
    prims = (8 + 8 + 40) / 3.0 if lean else 40
    tail = 3 * nface * r + 12 * r + 8 + 40 + 40 * 2.0 / 3.0 + 40 + prims + (20 if p.precision == 1 else 0)
    return {"face_x": face["x"], "face_y": face["y"], "face_z": face["z"], "visc_grad": visc, "stage_tail": tail}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """dram bytes per grid point per launch from the committed ncu summaries (profiles/traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [l.strip().split(",") for l in open(self.path) if l.strip()]
            sm = [float(r[1]) for r in rows if len(r) >= 9]
            mx = [float(r[2]) for r in rows if len(r) >= 9]
            reasons = set()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for r in rows:
                if len(r) < 9:
                    continue
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            if sm:
                out["sm_mhz"] = statistics.median(sm)
                out["sm_max_mhz"] = max(mx)
                out["samples"] = len(sm)
            out["reasons"] = sorted(reasons)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        return out


# ---------------------------------------------------------------------------------------------
def cpu_rate(p, steps: int, warm: int = 1, xyz=None, prims=None):
    """Oracle (CPU restatement, OpenMP over the host cores) grid-point updates per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle

    from ocfd_b200 import cases

    o = Oracle(p)
    if xyz is None:
        o.init_mesh()
    else:
        o.init_mesh(*xyz)
    o.init3d(cases.tgv_prims(o.p) if prims is None else prims)
    o.step(warm)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    n = p.nx * p.ny * p.nz
    o.close()
    return n * steps / dt / 1e9, dt


def data_kind(workload: str) -> str:
    if workload in WORKLOADS:
        return "synthetic (analytic Taylor-Green initial field)"
    if workload == "cylinder_weno7_char":
        return "synthetic (analytic body-fitted grid and uniform free stream)"
    return "synthetic (seeded isotropic-turbulence field)"


def cpu_case(workload: str):
    """(params, coordinates or None, interior primitives, sample description) of
    the oracle's CPU run: the workload itself, except for the 512^3 isotropic
    turbulence (about 80 GB of host memory and a minute per step on the oracle),
    which is sampled on 128^3 with the same set-up."""
    from ocfd_b200 import cases

    if workload == "hit512_hybrid_llf":
        p = cases.hit_params(128, re=1000.0, ma=1.0, dt=1e-3)
        return (p, cases.hit_coords(128), cases.hit_prims(128, mt=0.6, ma=1.0),
                "isotropic turbulence 128^3 with the same scheme (1/64 of the workload's points per step)")
    p, xyz, prims = make_case(workload, "fp64")
    return p, xyz, prims, f"the {grid_name(p)} workload itself (same scheme and grid)"


def run_reference(args):
    """The reference arm: the CPU restatement of the reference (oracle, all host
    threads) on the workload's own grid -- every step is one full time step of
    the same configuration as the GPU arm."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing

    cores = multiprocessing.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    p, xyz, prims, what = cpu_case(args.workload)
    rate, secs = cpu_rate(p, args.steps, warm=args.warmup, xyz=xyz, prims=prims)
    del prims, xyz
    ms = secs / args.steps * 1e3
    desc = WORKLOADS[args.workload][5] if args.workload in WORKLOADS else CASE_WORKLOADS[args.workload]
    sample = f"{args.steps} time steps of {what}, {p.nx * p.ny * p.nz} points a step, after {args.warmup} warm-up steps"
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": data_kind(args.workload),
        "config": {"workload": args.workload, "description": desc, "grid": grid_name(p), "dt": p.dt,
                   "precision": "fp64"},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def grid_name(p) -> str:
    return f"{p.nx}^3" if p.nx == p.ny == p.nz else f"{p.nx}x{p.ny}x{p.nz}"


# steps of the stated run of each workload: the horizon of the mixed-vs-FP64 errors
HORIZON = {"tgv256_omp6_char": 500, "tgv256_hybrid_char": 500, "tgv256_weno7": 500, "tgv64_weno7": 100,
           "hit512_hybrid_llf": 300, "cylinder_weno7_char": 2000}


# ---------------------------------------------------------------------------------------------
def _timed(s, steps: int, warmup: int, local: int, dist: bool):
    """W untimed steps, then K steps between CUDA events on the solver's stream
    (max over ranks), with the clocks sampled during the timed region."""
    import torch

    stream = torch.cuda.ExternalStream(s.stream, device=local)
    s.step(warmup, sync=True)  # includes graph capture
    if dist:
        import torch.distributed as tdist

        tdist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        s.step(steps, sync=False)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist:
        import torch.distributed as tdist

        t = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms = float(t.item())
    s.sync()  # raises if the run hit the reference's negative-temperature stop
    return ms, clk.summary()


def _kernels(s, n: int, peak: float, workload: str, precision: str):
    """Per-kernel CUDA-event split of 3 eager steps and the roofline of the dominant kernel."""
    prof = s.profile_steps(3)
    model = byte_model(s.p, s.metric_zero_mask())
    groups = {k: v for k, v in prof.items() if k in model}
    dom = max(groups, key=groups.get)
    t_launch = groups[dom] / 3.0 * 1e-3  # 3 launches per step
    achieved = model[dom] * n / t_launch / 1e9
    bpp = load_traffic().get(f"{workload}:{precision}:{dom}")
    return {"kernel": dom, "achieved": achieved, "frac": achieved / peak, "bytes_per_point": model[dom],
            "traffic": None if bpp is None else bpp * n,
            "kernel_ms_per_step": {k: round(v, 4) for k, v in prof.items()},
            "hbm_frac_by_kernel": {k: round(model[k] * n / (groups[k] / 3.0 * 1e-3) / 1e9 / peak, 3)
                                   for k in groups if groups[k] > 0}}


def _e2e(s, steps: int, dist: bool, local: int):
    """Same metric end to end through the C ABI with a host-owned state.  Headline
    mode: the host owns the conserved variables f (the reference's time-loop
    state); per step f is uploaded from pinned host memory, the primitives are
    derived from it on the device (comput_duvwT), one time step runs and f is
    downloaded.  Second mode: f and the haloed primitives both ways."""
    import ctypes as C

    import numpy as np
    import torch

    f_host = torch.empty(s.shape5, dtype=torch.float64, pin_memory=True).numpy()
    prim_host = [torch.empty(s.shape_h, dtype=torch.float64, pin_memory=True).numpy() for _ in range(5)]
    L = s.L
    dp = C.POINTER(C.c_double)
    fptr = f_host.ctypes.data_as(dp)
    parr = (dp * 5)(*[a.ctypes.data_as(dp) for a in prim_host])
    L.ocfd_gpu_download_state(s.h, fptr, C.cast(parr, C.c_void_p))
    istep, tt = s.time()
    if dist:
        import torch.distributed as tdist

        tdist.barrier()
    nneg = C.c_int(0)
    t0 = time.perf_counter()
    for _ in range(steps):
        L.ocfd_gpu_upload_state(s.h, fptr, None, istep, tt)
        L.ocfd_gpu_duvwt(s.h, C.byref(nneg))
        L.ocfd_gpu_step(s.h, 1, 0)
        L.ocfd_gpu_download_state(s.h, fptr, None)
        istep, tt = s.time()
    t_e2e = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _ in range(steps):
        L.ocfd_gpu_upload_state(s.h, fptr, C.cast(parr, C.c_void_p), istep, tt)
        L.ocfd_gpu_step(s.h, 1, 0)
        L.ocfd_gpu_download_state(s.h, fptr, C.cast(parr, C.c_void_p))
        istep, tt = s.time()
    t_full = time.perf_counter() - t0
    if dist:
        import torch.distributed as tdist

        t = torch.tensor([t_e2e, t_full], device=f"cuda:{local}", dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        t_e2e, t_full = float(t[0].item()), float(t[1].item())
    s.sync()
    n = s.nx * s.ny * s.nz
    return t_e2e, t_full, 5 * 8 * n, 5 * 8 * (n + int(np.prod(s.shape_h)))


def _history(s, prims, steps: int, every: int):
    """Restart from the initial field and run `steps` steps: kinetic energy
    (show_flow_msg) and enstrophy (ana_box) every `every` steps, and the final
    interior rho, u, v, w, p."""
    import numpy as np

    s.init3d(prims)
    ke, ens = [float(s.show_flow_msg()[1])], [float(s.ana_box()[13])]
    done = 0
    while done < steps:
        k = min(every, steps - done)
        s.step(k)
        done += k
        ke.append(float(s.show_flow_msg()[1]))
        ens.append(float(s.ana_box()[13]))
    _, pr = s.download_state()
    inner = (slice(4, -4),) * 3
    d, u, v, w, T = [np.ascontiguousarray(a[inner]) for a in pr]
    p = d * T / (s.p.gamma * s.p.ma * s.p.ma)  # p = rho T / (gamma Ma^2)
    return {"ke": np.array(ke), "enstrophy": np.array(ens), "rho": d, "vel": (u, v, w), "p": p}


def _errors(a: dict, b: dict) -> dict:
    """Errors of run a against run b (relative L2 and Linf on the interior)."""
    import numpy as np

    def rel(x, y):
        return abs(x - y) / abs(y)

    def l2(x, y):
        return float(np.sqrt(np.sum((x - y) ** 2) / np.sum(y ** 2)))

    def linf(x, y):
        return float(np.max(np.abs(x - y)) / np.max(np.abs(y)))

    du2 = sum(np.sum((x - y) ** 2) for x, y in zip(a["vel"], b["vel"]))
    u2 = sum(np.sum(y ** 2) for y in b["vel"])
    dumax = max(float(np.max(np.abs(x - y))) for x, y in zip(a["vel"], b["vel"]))
    umax = max(float(np.max(np.abs(y))) for y in b["vel"])
    return {"ke_rel": float(rel(a["ke"][-1], b["ke"][-1])),
            "ke_rel_max_history": float(np.max(np.abs(a["ke"] - b["ke"]) / np.abs(b["ke"]))),
            "enstrophy_rel": float(rel(a["enstrophy"][-1], b["enstrophy"][-1])),
            "enstrophy_rel_max_history": float(np.max(np.abs(a["enstrophy"] - b["enstrophy"]) /
                                                      np.abs(b["enstrophy"]))),
            "rho": {"l2_rel": l2(a["rho"], b["rho"]), "linf_rel": linf(a["rho"], b["rho"])},
            "u": {"l2_rel": float(np.sqrt(du2 / u2)), "linf_rel": dumax / umax},
            "p": {"l2_rel": l2(a["p"], b["p"]), "linf_rel": linf(a["p"], b["p"])}}


def run_ours(args):
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    if dist:
        import datetime

        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)

    from ocfd_b200.solver import Solver, footprint

    p, xyz, prims = make_case(args.workload, args.precision)
    n = p.nx * p.ny * p.nz
    peak, peak_kind = load_peaks()
    horizon = args.err_steps if args.err_steps is not None else HORIZON[args.workload]
    every = max(1, horizon // 10)

    def start(q):
        s = Solver(q, device=local)
        if xyz is None:
            s.init_mesh()
        else:
            s.init_mesh(*xyz)
        s.init3d(prims)
        return s

    # ---- the line's own precision: timed steps, kernel split, end to end
    s = start(p)
    ms, clocks = _timed(s, args.steps, args.warmup, local, dist)
    value = world * n * args.steps / (ms * 1e-3) / 1e9
    launches = args.steps * s.step_kernels()
    kern = _kernels(s, n, peak, args.workload, args.precision)
    K2 = max(1, min(args.steps, 5))
    t_e2e, t_full, bytes_f, bytes_state = _e2e(s, K2, dist, local)
    e2e = world * n * K2 / t_e2e / 1e9
    e2e_full = world * n * K2 / t_full / 1e9
    ke = s.show_flow_msg()[1]
    if not np.isfinite(ke):
        raise RuntimeError("non-finite kinetic energy: the run is invalid")
    fp_bytes = footprint(s.p)
    mixed = None
    if args.precision == "fp64" and not args.no_mixed:
        # ---- FP64 reference run over the error horizon, then the mixed-precision leg
        ref = _history(s, prims, horizon, every)
        s.close()
        pm = p.copy()
        pm.precision = 1
        sm = start(pm)
        ms_m, clocks_m = _timed(sm, args.steps, args.warmup, local, dist)
        value_m = world * n * args.steps / (ms_m * 1e-3) / 1e9
        launches_m = args.steps * sm.step_kernels()
        kern_m = _kernels(sm, n, peak, args.workload, "mixed")
        te_m, _, _, _ = _e2e(sm, K2, dist, local)
        hm = _history(sm, prims, horizon, every)
        sm.close()
        err = _errors(hm, ref)
        err["steps"] = horizon
        err["against"] = "the FP64 run of this line, same initial field and steps"
        mixed = {"value": value_m, "unit": UNIT, "ms_per_step": ms_m / args.steps, "mixed_over_fp64": value_m / value,
                 "dtype": "f32 flux/reconstruction/viscous, f64 state/metrics/primitive recovery",
                 "clocks": clocks_m, "gpu_launches": launches_m,
                 "e2e": {"value": world * n * K2 / te_m / 1e9, "unit": UNIT, "h2d_bytes_per_step": bytes_f,
                         "d2h_bytes_per_step": bytes_f},
                 "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s", **kern_m},
                 "error_vs_fp64": err}
    else:
        s.close()
    del prims, xyz
    served = None
    if args.workload in WORKLOADS and not args.no_serve and world == 1:
        served = served_leg()

    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu and world == 1:
            import multiprocessing

            cores = multiprocessing.cpu_count()
            os.environ.setdefault("OMP_NUM_THREADS", str(cores))
            # about 10-30 s of the host's cores on the workload's own grid: 1 warm-up step,
            # then enough full steps for about 10 s
            q, qxyz, qprims, what = cpu_case(args.workload)
            rate, secs = cpu_rate(q, 1, warm=1, xyz=qxyz, prims=qprims)
            nst = int(min(40, max(2, 10.0 / max(secs, 1e-3))))
            rate, secs = cpu_rate(q, nst, warm=1, xyz=qxyz, prims=qprims)
            del qprims, qxyz
            cpu = {"value": rate, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
                   "sample": f"{nst} time steps of {what} on the oracle after 1 warm-up step ({secs:.1f} s)"}
        desc = WORKLOADS[args.workload][5] if args.workload in WORKLOADS else CASE_WORKLOADS[args.workload]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32 flux / f64 state",
            "data": data_kind(args.workload),
            "config": {"workload": args.workload, "description": desc, "grid": grid_name(p), "dt": p.dt,
                       "precision": args.precision, "parallelism": f"replicas x{world}",
                       "l2": (f"device state {fp_bytes / 2**20:.0f} MiB (conserved and primitive fields, "
                              f"metrics, face and viscous fluxes), all read every step: larger than the "
                              f"126 MB L2, no flush")},
            "clocks": clocks,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": bytes_f, "d2h_bytes_per_step": bytes_f,
                    "mode": "host-owned conserved state f: upload f, primitives derived on the device "
                            "(comput_duvwT), one step, download f",
                    "with_primitives": {"value": e2e_full, "h2d_bytes_per_step": bytes_state,
                                        "d2h_bytes_per_step": bytes_state,
                                        "mode": "upload f + haloed primitives, one step, download both"}},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_kind": peak_kind, **kern,
                         "note": "the face kernels are FP64-pipe (FP64) or issue (FP32) bound, not HBM bound"},
            "mixed": mixed,
            "served": served,
            "cpu_baseline": cpu,
            "kinetic_energy": ke,
        }
        print(json.dumps(line), flush=True)
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()
    return 0


def served_leg(count: int = 64, rate: float = 16.0, steps=(100, 300)) -> dict:
    """A compact served stream for the default bench line: `count` seeded Poisson
    requests (TGV / isotropic turbulence, 32^3-128^3, mixed precision, served with
    continuous batching), against the same requests solved one after another in
    FP64 and in mixed precision.  Host clock (time to result is wall time)."""
    from concurrent.futures import ThreadPoolExecutor

    from ocfd_b200 import serving

    reqs = serving.make_stream(count, rate=rate, seed=20261204, steps=steps)
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
        prepared = list(ex.map(lambda r: serving.request_setup(r, True), reqs))
    payloads = {r.rid: x for r, x in zip(reqs, prepared)}
    served = serving.Server(mixed=True).run(reqs, realtime=True, payloads=payloads)
    seq = serving.run_sequential(reqs, mixed=False, payloads=payloads)
    seq_m = serving.run_sequential(reqs, mixed=True, payloads=payloads)
    pick = lambda d: {k: d[k] for k in ("gpts_per_s", "p50_s", "p99_s", "span_s")}
    return {"requests": count, "rate_per_s": rate, "steps": list(steps),
            "work_gpt_steps": int(sum(r.n ** 3 * r.steps for r in reqs)),
            "served_mixed": pick(served) | {"rounds": served["rounds"]},
            "sequential_fp64": pick(seq), "sequential_mixed": pick(seq_m),
            "served_over_sequential_fp64": served["gpts_per_s"] / seq["gpts_per_s"],
            "served_over_sequential_mixed": served["gpts_per_s"] / seq_m["gpts_per_s"],
            "note": "results bit-identical alone and in the mix; the full 256-request stream with errors "
                    "against FP64 is the --serve mode"}


def run_serve(args):
    """Served mixed-precision stream (continuous batching) against sequential plain
    FP64 solves of the same requests.  The error of the served results against
    the FP64 ones is stated on a sample of requests beside the predictability
    floor of each flow: the FP64 solve from an initial field perturbed by one
    FP32 rounding (relative 2^-24), since at these Reynolds numbers and step
    counts the flows are chaotic and any rounding difference grows."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    from ocfd_b200 import serving

    reqs = serving.make_stream(args.requests, rate=args.rate, seed=20261203)
    sample = [r.rid for r in reqs[:: max(1, len(reqs) // 16)]]
    # the requests arrive with their initial fields (prepared before the stream starts)
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
        prepared = list(ex.map(lambda r: serving.request_setup(r, True), reqs))
    payloads = {r.rid: x for r, x in zip(reqs, prepared)}
    srv = serving.Server(mixed=True, round_steps=args.round_steps, keep=sample)
    served = srv.run(reqs, realtime=True, payloads=payloads)
    seq = serving.run_sequential(reqs, mixed=False, keep=sample, payloads=payloads)
    # the same requests solved one after another in mixed precision: the served
    # stream against it is the gain of batching alone
    seq_m = serving.run_sequential(reqs, mixed=True, payloads=payloads)

    inner = (slice(4, -4),) * 3

    def errors(a_state, a_E0, b_state, b_E0, ma):
        (fa, pa), (fb, pb) = a_state, b_state
        rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
        pr = lambda P: P[0][inner] * P[4][inner] / (1.4 * ma * ma)
        return {"ke": abs(a_E0[1] - b_E0[1]) / abs(b_E0[1]), "rho": rel(pa[0][inner], pb[0][inner]),
                "u": max(rel(pa[q][inner], pb[q][inner]) for q in (1, 2, 3)), "p": rel(pr(pa), pr(pb))}

    mixed_err, floor_err = [], []
    rng = np.random.default_rng(5)
    for rid in sample:
        r = reqs[rid]
        b = seq["results"][rid]
        a = served["results"][rid]
        mixed_err.append(errors(a.state, a.E0, b.state, b.E0, r.ma))
        p, xyz, prims = payloads[rid]
        p = p.copy()
        p.precision = 0
        pert = [prims[0]] + [q * (1.0 + 2.0 ** -24 * rng.standard_normal(q.shape)) for q in prims[1:]]
        s = serving._start(p, xyz, pert, 0)
        s.step(r.steps)
        floor_err.append(errors(s.download_state(), s.show_flow_msg().tolist(), b.state, b.E0, r.ma))
        s.close()
    agg = lambda L: {f"{k}_rel_max": max(e[k] for e in L) for k in ("ke", "rho", "u", "p")} | {
        f"{k}_rel_median": float(np.median([e[k] for e in L])) for k in ("ke", "u")}
    # per request at a short horizon (before the chaotic growth of rounding
    # differences): mixed against FP64 after HS steps, both alone -- a served
    # result is bit-identical to the same request solved alone
    HS = 20
    short = []
    for rid in sample:
        p, xyz, prims = payloads[rid]
        out = []
        for prec in (1, 0):
            q = p.copy()
            q.precision = prec
            s = serving._start(q, xyz, prims, 0)
            s.step(HS)
            out.append((s.download_state(), s.show_flow_msg().tolist()))
            s.close()
        short.append(errors(out[0][0], out[0][1], out[1][0], out[1][1], reqs[rid].ma))
    work = sum(r.n ** 3 * r.steps for r in reqs)
    line = {
        "metric": "served stream: aggregate GPts/s and p50/p99 time-to-result, mixed precision, continuous batching",
        "mode": "serve", "requests": len(reqs), "rate_per_s": args.rate, "work_gpt_steps": work,
        "data": "synthetic (seeded Poisson stream of TGV / isotropic-turbulence requests, sizes 32^3-128^3)",
        "served_mixed": {k: served[k] for k in ("gpts_per_s", "p50_s", "p99_s", "span_s", "rounds", "batched_rounds",
                                                 "persistent_rounds",
                                                 "max_active")},
        "sequential_fp64": {k: seq[k] for k in ("gpts_per_s", "p50_s", "p99_s", "span_s", "wall_s")},
        "sequential_mixed": {k: seq_m[k] for k in ("gpts_per_s", "p50_s", "p99_s", "span_s", "wall_s")},
        "throughput_ratio": served["gpts_per_s"] / seq["gpts_per_s"],
        "throughput_ratio_vs_sequential_mixed": served["gpts_per_s"] / seq_m["gpts_per_s"],
        "error_vs_fp64_at_20_steps": {"sample": len(sample), **agg(short)},
        "error_vs_fp64": {"sample": len(sample), **agg(mixed_err)},
        "fp64_perturbed_2^-24_vs_fp64": agg(floor_err),
        "scheme": "WENO7 flux-vector, SW, CD6; dt at CFL 0.5 from the initial field",
        "grouping": f"instances of {srv.solo_min}^3 points and more on their own step graphs, smaller ones batched",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args):
    """Steady-state throughput of batched mixed-precision steps (the serving
    path's WENO7 flux-vector form) per member set, in both launch modes (one
    launch per kernel and RK stage; one persistent launch per stage), beside
    the members stepped one after another alone.  Host clock over --steps steps
    after --warmup (synchronised on both sides), GPts/s."""
    import time

    from ocfd_b200 import serving
    from ocfd_b200.solver import Batch

    def members(sizes):
        out = []
        for q, n in enumerate(sizes):
            r = serving.Request(rid=q, kind="tgv" if q % 2 == 0 else "hit", n=n, re=1600.0, ma=0.3,
                                steps=10 ** 6, arrival=0.0, seed=1000 + q)
            p, xyz, prims = serving.request_setup(r, True)
            out.append(serving._start(p, xyz, prims, 0))
        return out

    sets = {"64 x 32^3": [32] * 64, "19 x 48^3": [48] * 19, "8 x 64^3": [64] * 8, "2 x 96^3": [96] * 2,
            "1 x 128^3": [128], "12 ragged 32^3-128^3": [32, 48, 64, 96, 128, 32, 48, 64, 32, 48, 64, 128]}
    res = {}
    for name, sizes in sets.items():
        ms = members(sizes)
        pts = sum(n ** 3 for n in sizes)
        row = {}
        for mode in (False, True):
            b = Batch(ms)
            b.set_persistent(mode)
            b.step(args.warmup)
            t0 = time.perf_counter()
            b.step(args.steps)
            row["persistent" if mode else "per_kernel"] = pts * args.steps / (time.perf_counter() - t0) / 1e9
            b.close()
        for s in ms:
            s.step(args.warmup)
        t0 = time.perf_counter()
        for s in ms:
            s.step(args.steps)  # each alone on its own step graph, one after another
        row["single"] = pts * args.steps / (time.perf_counter() - t0) / 1e9
        for s in ms:
            s.close()
        res[name] = {k: round(v, 4) for k, v in row.items()}
    print(json.dumps({"metric": "batched mixed WENO7 steady state", "unit": "GPts/s", "steps": args.steps,
                      "warmup": args.warmup, "sets": res}), flush=True)
    return 0


def run_history(args):
    """Kinetic-energy, dissipation-rate (-dK/dt) and enstrophy histories of the
    256^3 characteristic TGV runs (OMP6 and hybrid): the GPU production build
    against the oracle over the first `--hist-oracle-steps` steps (the oracle
    needs seconds per step at this size), and the GPU alone over the full
    `--hist-steps` steps."""
    import numpy as np

    from ocfd_b200.solver import Solver

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle

    from ocfd_b200 import cases

    every = args.hist_every
    out = {"mode": "history", "grid": "256^3", "dt": WORKLOADS["tgv256_omp6_char"][4], "every": every,
           "data": "synthetic (analytic Taylor-Green initial field)"}
    for wl in ("tgv256_omp6_char", "tgv256_hybrid_char"):
        rec = {}
        for kind in ("gpu", "oracle"):
            p = make_params(wl, "fp64")
            steps = args.hist_steps if kind == "gpu" else args.hist_oracle_steps
            s = Solver(p) if kind == "gpu" else Oracle(p)
            s.init_mesh()
            s.init3d(cases.tgv_prims(s.p))
            t, ke, ens = [0.0], [float(s.show_flow_msg()[1])], [float(s.ana_box()[13])]
            done = 0
            while done < steps:
                k = min(every, steps - done)
                s.step(k)
                done += k
                t.append(done * p.dt)
                ke.append(float(s.show_flow_msg()[1]))
                ens.append(float(s.ana_box()[13]))
            s.close()
            t, ke = np.array(t), np.array(ke)
            eps = -(ke[1:] - ke[:-1]) / (t[1:] - t[:-1])
            rec[kind] = {"t": t.tolist(), "ke": ke.tolist(), "eps": eps.tolist(), "enstrophy": ens}
        g, o = rec["gpu"], rec["oracle"]
        m = len(o["ke"])
        rel = lambda a, b: float(np.max(np.abs(np.array(a) - np.array(b)) / np.maximum(np.abs(np.array(b)), 1e-300)))
        out[wl] = {"gpu_steps": args.hist_steps, "oracle_steps": args.hist_oracle_steps,
                   "ke_rel_max": rel(g["ke"][:m], o["ke"]), "eps_rel_max": rel(g["eps"][:m - 1], o["eps"]),
                   "enstrophy_rel_max": rel(g["enstrophy"][:m], o["enstrophy"]), "gpu": g, "oracle": o}
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tgv256_omp6_char", choices=list(WORKLOADS) + list(CASE_WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg of an FP64 line")
    ap.add_argument("--no-serve", action="store_true", help="skip the compact served-stream leg")
    ap.add_argument("--err-steps", type=int, default=None,
                    help="horizon of the mixed-vs-FP64 errors (default: the workload's stated step count)")
    ap.add_argument("--serve", action="store_true", help="served request stream instead of the step benchmark")
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--rate", type=float, default=8.0, help="Poisson arrival rate, requests per second")
    ap.add_argument("--round-steps", type=int, default=25)
    ap.add_argument("--batched", action="store_true",
                    help="steady-state batched throughput per member set (both launch modes) instead")
    ap.add_argument("--history", action="store_true", help="kinetic-energy / dissipation histories vs the oracle")
    ap.add_argument("--hist-steps", type=int, default=500)
    ap.add_argument("--hist-oracle-steps", type=int, default=20)
    ap.add_argument("--hist-every", type=int, default=5)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.serve:
        return run_serve(args)
    if args.history:
        return run_history(args)
    if args.batched:
        return run_batched(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
