"""Serving loop: a stream of Navier-Stokes solve requests on one GPU with
continuous batching.

Requests (Taylor-Green or isotropic-turbulence instances of different grid
sizes, Reynolds and Mach numbers and step counts) arrive over time.  The loop
admits a waiting request as soon as a slot, device memory (by the instance's
exact footprint) and room under the cap of grid points in flight are free, keeps every admitted instance's state on
the device, and advances all active instances together in rounds of at most
`round_steps` steps with one batched launch per kernel and RK stage
(ocfd_batch_*).  A request that finishes frees its slot and memory at the end
of its round, and requests that arrived meanwhile join at the next round.  Each
result is bit-identical to the same request solved alone (the batched kernels
compute every instance exactly as the single-instance kernels do).

The reference runs one case per process and has no serving layer; this module
is the host side of the ensemble entry points.
"""
from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import cases
from .params import SCHEME_WENO7, SPLIT_SW
from .solver import Batch, Solver, footprint, set_parameters

SIZES = (32, 48, 64, 96, 128)


@dataclass
class Request:
    rid: int
    kind: str            # "tgv" or "hit"
    n: int               # grid points per direction
    re: float
    ma: float
    steps: int
    arrival: float       # seconds after the start of the stream
    seed: int = 0


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    points: int
    E0: list
    state: tuple | None = None  # (f, prims) when kept

    @property
    def time_to_result(self) -> float:
        return self.finished - self.arrival


def make_stream(count: int, rate: float, seed: int = 20261203, sizes=SIZES, steps=(200, 1000),
                re=(400.0, 3200.0), ma=(0.1, 0.5)) -> list[Request]:
    """Seeded Poisson arrivals (rate per second) of TGV / HIT requests with grid
    sizes drawn uniformly from `sizes`, Re and Ma uniform, steps uniform."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for q in range(count):
        t += float(rng.exponential(1.0 / rate)) if rate > 0 else 0.0
        out.append(Request(rid=q, kind="tgv" if rng.random() < 0.5 else "hit", n=int(rng.choice(sizes)),
                           re=float(rng.uniform(*re)), ma=float(rng.uniform(*ma)),
                           steps=int(rng.integers(steps[0], steps[1] + 1)), arrival=t,
                           seed=int(rng.integers(1, 2 ** 31 - 1))))
    return out


def request_setup(req: Request, mixed: bool):
    """Parameters, coordinates (None = box grid) and interior primitives of a
    request.  Scheme: WENO7 flux-vector form, Steger-Warming, CD6 viscous terms
    (the same for both kinds so that all requests share one batched launch);
    dt from the initial field at CFL 0.5: 0.5 h / max(|u|+|v|+|w| + c)."""
    n = req.n
    h = 2.0 * math.pi / n
    if req.kind == "tgv":
        p = cases.tgv_params(n, scheme=SCHEME_WENO7, character=0, split=SPLIT_SW, ma=req.ma, re=req.re)
        prims = cases.tgv_prims(p)
        xyz = None
    else:
        # the random field is periodic, so it is laid on the same box grid as TGV
        p = cases.tgv_params(n, scheme=SCHEME_WENO7, character=0, split=SPLIT_SW, ma=req.ma, re=req.re)
        prims = cases.hit_prims(n, mt=0.6, ma=req.ma, seed=req.seed)
        xyz = None
    vmax = float(np.max(np.abs(prims[1]) + np.abs(prims[2]) + np.abs(prims[3])
                        + np.sqrt(prims[4]) / req.ma))
    p.dt = 0.5 * h / vmax
    p.end_time = p.dt * req.steps
    p.precision = 1 if mixed else 0
    return p, xyz, prims


def _start(p, xyz, prims, device):
    s = Solver(p, device=device)
    if xyz is None:
        s.init_mesh()
    else:
        s.init_mesh(*xyz)
    s.init3d(prims)
    return s


class Server:
    """Continuous-batching request loop on one device."""

    def __init__(self, device: int = 0, mixed: bool = True, hbm_budget: int | None = None, max_slots: int = 96,
                 round_steps: int = 25, keep=(), prefetch: int = 16, max_points: int = 6_000_000,
                 solo_min: int = 96, launch_mode: str = "timed"):
        from . import _lib

        self.device = device
        self.mixed = mixed
        self.max_slots = max_slots
        self.round_steps = round_steps
        self.keep = set(keep)
        self.prefetch = prefetch
        # grid points in flight: enough to fill the GPU (about 2M points already
        # run at full rate), few enough that requests finish in arrival order
        # rather than all at the end (lower time to result)
        self.max_points = max_points
        # instances of at least solo_min^3 points advance on their own captured
        # step graphs (single-instance kernels, concurrently on their own
        # streams): measured faster than their part of a batched launch; the
        # smaller ones share the batched launches, which run several of them at
        # once where alone each would leave most of the GPU idle
        self.solo_min = solo_min
        # batched launch mode: "timed" (each new set of grid sizes times both modes
        # on its first round and keeps the faster), "per_kernel" or "persistent"
        if launch_mode not in ("timed", "per_kernel", "persistent"):
            raise ValueError(f"launch_mode {launch_mode!r}")
        self.launch_mode = launch_mode
        self.hbm_budget = hbm_budget if hbm_budget is not None else _free_device_memory(device) * 85 // 100
        # per set of grid sizes: the face tile variants and the launch mode (one
        # launch per kernel or one persistent launch per stage), chosen by timing
        # on the first batch of those sizes and reused
        self.tiles: dict[tuple, tuple] = {}
        _lib.lib()  # fail loudly here if the library is not built

    def run(self, requests: list[Request], realtime: bool = True, payloads: dict | None = None) -> dict:
        """Serve the stream.  realtime=True replays the arrival times against the
        wall clock; False admits every request as if it had arrived at t=0.
        payloads: rid -> request_setup() result, when the requests arrive with
        their initial fields; otherwise a worker thread prepares them ahead."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        prepared: dict[int, tuple] = dict(payloads) if payloads else {}
        ready = threading.Condition()
        th = None
        if not payloads:
            work: queue.Queue = queue.Queue()
            for r in reqs:
                work.put(r)

            def worker():
                while True:
                    try:
                        r = work.get_nowait()
                    except queue.Empty:
                        return
                    item = request_setup(r, self.mixed)
                    with ready:
                        prepared[r.rid] = item
                        ready.notify_all()
                        while len(prepared) > self.prefetch:  # bound host memory
                            ready.wait(0.05)

            th = threading.Thread(target=worker, daemon=True)
            th.start()

        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        arrival = (lambda r: r.arrival) if realtime else (lambda r: 0.0)
        waiting = list(reqs)
        active: list[dict] = []   # admitted, with steps left to enqueue
        results: dict[int, Result] = {}
        used = 0
        batch = None
        members_key = None
        in_flight = None          # (batch, members finishing with it, stale batch or None) of the enqueued round
        rounds = batched_rounds = persistent_rounds = max_active = 0
        while waiting or active or in_flight:
            # 1. enqueue the next round of the active instances (asynchronous; on
            # the GPU it follows the round in flight, which is not waited for)
            run = [a for a in active if a["left"] > 0]
            flight = None
            if run:
                k = min(self.round_steps, min(a["left"] for a in run))
                solo = [a for a in run if a["req"].n >= self.solo_min]
                grouped = [a for a in run if a["req"].n < self.solo_min]
                for a in solo:
                    a["s"].step(k, sync=False)
                key = tuple(a["req"].rid for a in grouped)
                stale = None
                tuned_now = None
                if grouped and key != members_key:
                    stale = batch  # closed once its round has been retired
                    batch = Batch([a["s"] for a in grouped])
                    members_key = key
                    if self.launch_mode != "timed":
                        batch.set_persistent(self.launch_mode == "persistent")
                    sizes = tuple(sorted({a["req"].n for a in grouped}))
                    if sizes in self.tiles:
                        variants, mode = self.tiles[sizes]
                        batch.set_tiles(variants)
                        if mode is not None and self.launch_mode == "timed":
                            batch.set_persistent(mode == 2)
                        else:
                            tuned_now = sizes  # the launch mode is still to be timed
                    else:
                        tuned_now = sizes
                rounds += 1
                if grouped:
                    batch.step(k, sync=False)
                    fused, variants = batch.info()
                    batched_rounds += 1 if fused else 0
                    persistent_rounds += 1 if batch.mode() == 2 else 0
                    if tuned_now is not None and fused:
                        # the launch mode is kept once it was timed (a round of at least four steps)
                        self.tiles[tuned_now] = (variants, batch.mode() if batch.mode_times() is not None else None)
                for a in run:
                    a["left"] -= k
                max_active = max(max_active, len(run))
                flight = (batch if grouped else None, [a for a in run if a["left"] == 0], stale)
            # 2. while it runs: admit arrived requests (FIFO) into free slots and memory
            new: list[dict] = []
            now = clock()
            busy = len(run) > 0 or in_flight is not None
            while waiting and arrival(waiting[0]) <= now and len(active) + len(new) < self.max_slots:
                r = waiting[0]
                with ready:
                    while r.rid not in prepared:
                        ready.wait(0.05)
                    p, xyz, prims = prepared[r.rid]
                need = footprint(set_parameters(p))
                pts = sum(a["req"].n ** 3 for a in active + new if a["left"] > 0)
                if (busy or new) and (used + need > self.hbm_budget or pts + r.n ** 3 > self.max_points):
                    break
                with ready:
                    prepared.pop(r.rid)
                    ready.notify_all()
                waiting.pop(0)
                s = _start(p, xyz, prims, self.device)
                used += need
                new.append({"req": r, "s": s, "left": r.steps, "admitted": clock(), "bytes": need})
            # 3. retire the previous round: results of the instances that finished
            # with it (their streams follow it; the round enqueued above keeps
            # the GPU busy meanwhile), their slots and memory freed
            if in_flight is not None:
                ob, fin, ostale = in_flight
                for a in fin:
                    r, s = a["req"], a["s"]
                    s.sync()  # negative-temperature status of the finished request
                    E0 = s.show_flow_msg().tolist()
                    st = s.download_state() if r.rid in self.keep else None
                    results[r.rid] = Result(rid=r.rid, arrival=arrival(r), admitted=a["admitted"], finished=clock(),
                                            steps=r.steps, points=r.n ** 3, E0=E0, state=st)
                if ostale is not None:
                    ostale.close()
                if ob is not None and ob is not batch and (flight is None or flight[2] is not ob):
                    ob.close()
                if fin:
                    done = {id(a) for a in fin}
                    for a in fin:
                        a["s"].close()
                        used -= a["bytes"]
                    active = [a for a in active if id(a) not in done]
            in_flight = flight
            active = active + new
            if not run and in_flight is None and not new and waiting:
                time.sleep(max(0.0, min(arrival(waiting[0]) - clock(), 0.5)))
        if batch is not None:
            batch.close()
        if th is not None:
            th.join(timeout=1.0)
        span = max(r.finished for r in results.values()) - min(r.arrival for r in results.values())
        work_pts = sum(r.points * r.steps for r in results.values())
        ttr = np.array([r.time_to_result for r in results.values()])
        return {"results": results, "span_s": span, "gpts_per_s": work_pts / span / 1e9,
                "p50_s": float(np.percentile(ttr, 50)), "p99_s": float(np.percentile(ttr, 99)),
                "rounds": rounds, "batched_rounds": batched_rounds, "persistent_rounds": persistent_rounds,
                "max_active": max_active}


def run_sequential(requests: list[Request], mixed: bool = False, device: int = 0, keep=(),
                   payloads: dict | None = None) -> dict:
    """The same requests solved one after another, each alone (ocfd_gpu_step),
    in arrival order; time to result from the replayed arrival times.  The
    host-side initial fields are not timed (payloads, or prepared per request
    before its clock starts)."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    results: dict[int, Result] = {}
    t0 = time.perf_counter()
    busy = 0.0
    for r in reqs:
        if payloads:
            p, xyz, prims = payloads[r.rid]
            p = p.copy()
            p.precision = 1 if mixed else 0
        else:
            p, xyz, prims = request_setup(r, mixed)
        # the GPU is free at max(arrival, previous finish); setup is host work
        start_wall = time.perf_counter()
        s = _start(p, xyz, prims, device)
        s.step(r.steps)
        E0 = s.show_flow_msg().tolist()
        st = s.download_state() if r.rid in keep else None
        s.close()
        dur = time.perf_counter() - start_wall
        start = max(r.arrival, busy)
        busy = start + dur
        results[r.rid] = Result(rid=r.rid, arrival=r.arrival, admitted=start, finished=busy, steps=r.steps,
                                points=r.n ** 3, E0=E0, state=st)
    wall = time.perf_counter() - t0
    span = max(x.finished for x in results.values()) - min(x.arrival for x in results.values())
    work_pts = sum(x.points * x.steps for x in results.values())
    ttr = np.array([x.time_to_result for x in results.values()])
    busy_total = sum(x.finished - x.admitted for x in results.values())
    return {"results": results, "span_s": span, "gpts_per_s": work_pts / busy_total / 1e9, "wall_s": wall,
            "p50_s": float(np.percentile(ttr, 50)), "p99_s": float(np.percentile(ttr, 99))}


def _free_device_memory(device: int) -> int:
    """Free device memory in bytes (cudaMemGetInfo through the CUDA runtime the
    library links against)."""
    import ctypes as C
    try:
        cudart = C.CDLL("libcudart.so.12")
    except OSError:
        return 64 << 30
    free, total = C.c_size_t(), C.c_size_t()
    if cudart.cudaSetDevice(device) != 0 or cudart.cudaMemGetInfo(C.byref(free), C.byref(total)) != 0:
        return 64 << 30
    return int(free.value)
