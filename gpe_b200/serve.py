"""Serving loop: a stream of Gross-Pitaevskii solve requests served by one
GPU with continuous batching.

Requests arrive over time (Poisson), are admitted into a Pool -- shortest
job first among those that have arrived, as long as their state fits in the
HBM budget and the sites in flight stay under a cap -- join the running
batch at the next chunk boundary, and leave with their final state when
done.  Latency of a request
= completion time - arrival time (host clock).  Nothing here waits for the
batch to drain before admitting new work.
"""
from __future__ import annotations

import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import ic
from .pool import Pool
from .solver import RunParams


@dataclass
class Request:
    tag: int
    arrival_s: float
    params: RunParams
    nsteps: int
    ic_kind: str          # "ring" | "line" | "random_phase"
    seed: int
    ic_arg: float = 0.0   # ring radius / random-phase cutoff

    @property
    def sites(self) -> int:
        p = self.params
        return p.nx * p.ny * p.nz


def initial_state(req: Request) -> np.ndarray:
    """Per-request initial state from its seed (host side)."""
    p = req.params
    if req.ic_kind == "ring":
        psi = ic.vortex_ring(p, "xy", r0=req.ic_arg)
    elif req.ic_kind == "line":
        psi = ic.vortex_line_pade(p, dir="z")
        if p.omx or p.omy or p.omz:
            psi = ic.fermi(p) * psi
    else:
        psi = ic.random_phase(p, seed=req.seed, kc=req.ic_arg)
    return psi.astype(np.complex64) if p.storage == "c64" else psi


def device_ic(req: Request):
    """The request's initial state as a device-side IC spec (no host array,
    no host-to-device copy)."""
    p = req.params
    if req.ic_kind == "ring":
        return ic.device_spec("ring", ring=dict(plane="xy", r0=req.ic_arg))
    if req.ic_kind == "line":
        if p.omx or p.omy or p.omz:
            return ic.device_spec("fermi", "line_pade")
        return ic.device_spec("line_pade")
    return ic.device_spec("random_phase", seed=req.seed, kc=req.ic_arg)


def make_requests(n: int, rate_per_s: float = 20.0, seed: int = 2024,
                  sizes=tuple(range(48, 257, 16)), steps=(200, 5000)) -> list[Request]:
    """Synthetic request stream: Poisson arrivals; cubic sizes uniform in
    `sizes`; steps uniform in [steps]; RK4 or RKF45; order 2 or 4; V = 0 or
    an isotropic trap with omega uniform in [0.02, 0.1]; initial state ring /
    line / random phase from a per-request seed; FP64 or FP32 storage."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate_per_s)
        nn = int(rng.choice(sizes))
        trap = bool(rng.integers(0, 2))
        om = float(rng.uniform(0.02, 0.1)) if trap else 0.0
        scheme = "rk4" if rng.integers(0, 2) == 0 else "rk45"
        kind = ("ring", "line", "random_phase")[int(rng.integers(0, 3))]
        if kind == "random_phase":
            trap, om = False, 0.0
        h = 0.25 * (nn - 1)  # dx = 0.5
        mu = 1.0
        if trap:
            # Thomas-Fermi radius covers the box: mu = 1 + V at the corner
            mu = 1.0 + 0.5 * om * om * 3 * h * h
        rp = RunParams(nx=nn, ny=nn, nz=nn, xr=h, yr=h, zr=h, tau=0.01 if scheme == "rk4" else 0.005,
                       scheme=scheme, eqn_to_solve=4, bcs=1 if kind == "random_phase" else 2,
                       order=int(rng.choice([2, 4])), g=1.0, mu=mu, omx=om, omy=om, omz=om,
                       storage="c128" if rng.integers(0, 2) == 0 else "c64")
        arg = float(rng.uniform(2.0, 6.0)) if kind == "ring" else float(rng.uniform(1.0, 2.0))
        out.append(Request(k, t, rp, int(rng.integers(steps[0], steps[1] + 1)), kind, int(rng.integers(1 << 30)),
                           arg))
    return out


@dataclass
class ServeReport:
    latencies_s: dict = field(default_factory=dict)
    site_updates: int = 0
    wall_s: float = 0.0
    max_active: int = 0
    rejected_admissions: int = 0

    def summary(self) -> dict:
        lat = np.array(sorted(self.latencies_s.values()))
        return {"requests": int(len(lat)), "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "site_updates_per_s": self.site_updates / self.wall_s if self.wall_s else None,
                "wall_s": self.wall_s, "max_active": self.max_active,
                "deferred_admissions": self.rejected_admissions}


def serve(requests: list[Request], budget_bytes: int, chunk: int = 50, realtime: bool = True,
          prep_threads: int = 4, device_ics: bool = True, max_active_sites: int = 48 << 20,
          on_result=None, policy: str = "sjf") -> ServeReport:
    """Run the request stream through one Pool.  With realtime=True a request
    becomes visible at its arrival time on the host clock; every loop turn
    admits what has arrived and fits, advances the batch by up to `chunk`
    steps, and collects finished solves.  device_ics=True builds each
    initial state on the GPU at admission; False prepares it on host
    threads and copies it in.  on_result(request, result), if given, sees
    every finished solve before its result buffer is reused.  policy (device
    ICs): "sjf" admits the arrived requests with the least work (sites x
    steps) first, "fcfs" in arrival order; either way up to
    max_active_sites grid sites in flight."""
    if device_ics:
        return _serve_device_ics(requests, budget_bytes, chunk, realtime, max_active_sites, on_result, policy)
    pool = Pool(budget_bytes)
    rep = ServeReport()
    pending = sorted(requests, key=lambda r: r.arrival_s)
    # initial states are prepared on host threads as requests arrive (numpy
    # releases the GIL in its FFT and array kernels); a request is admitted
    # once its state is ready and fits in the budget
    prep = ThreadPoolExecutor(max_workers=prep_threads)
    waiting: list[tuple[Request, Future]] = []
    by_tag = {r.tag: r for r in requests}
    t0 = time.perf_counter()
    active = 0
    nxt = 0
    while nxt < len(pending) or waiting or active:
        now = time.perf_counter() - t0
        while nxt < len(pending) and (not realtime or pending[nxt].arrival_s <= now):
            waiting.append((pending[nxt], prep.submit(initial_state, pending[nxt])))
            nxt += 1
        still = []
        for req, fut in waiting:
            if not fut.done():
                still.append((req, fut))
            elif pool.submit(req.params, fut.result(), req.nsteps, req.tag):
                active += 1
            else:
                rep.rejected_admissions += 1
                still.append((req, fut))
        waiting = still
        if active == 0:
            time.sleep(0.002)
            continue
        rep.max_active = max(rep.max_active, active)
        active = pool.step(chunk)
        done_t = time.perf_counter() - t0
        for r in pool.poll():
            req = by_tag[r.tag]
            rep.latencies_s[r.tag] = done_t - req.arrival_s
            rep.site_updates += req.sites * r.steps
            if on_result:
                on_result(req, r)
    rep.wall_s = time.perf_counter() - t0
    prep.shutdown()
    pool.close()
    return rep


class ResultBuffers:
    """Page-locked result buffers reused across requests of the same shape:
    a finished solve's state lands by DMA, and the buffer goes back to the
    free list once the result has been handed on."""

    def __init__(self):
        self._free: dict[tuple, list[np.ndarray]] = {}

    def get(self, shape, dtype) -> np.ndarray:
        key = (tuple(shape), np.dtype(dtype).str)
        lst = self._free.get(key)
        if lst:
            return lst.pop()
        from . import _lib as L

        return L.pinned_empty(shape, dtype)

    def put(self, arr: np.ndarray) -> None:
        self._free.setdefault((arr.shape, arr.dtype.str), []).append(arr)


def _storage_dtype(params) -> np.dtype:
    return np.dtype(np.complex64 if params.storage == "c64" else np.complex128)


def _serve_device_ics(requests, budget_bytes, chunk, realtime, max_active_sites, on_result=None,
                      policy: str = "sjf") -> ServeReport:
    """Admission is bounded by the HBM budget and by max_active_sites: enough
    grid sites in flight to keep the GPU's memory system busy, no more, so
    that admitted requests are not slowed by every later arrival.  Among the
    arrived requests, "sjf" admits the one with the least work first (a
    solve in the pool runs to completion, so this is shortest-job-first
    without preemption): short requests no longer queue behind long ones,
    which is what sets the median latency under load; "fcfs" keeps arrival
    order."""
    if policy not in ("sjf", "fcfs"):
        raise ValueError("policy must be 'sjf' or 'fcfs'")
    pool = Pool(budget_bytes)
    rep = ServeReport()
    bufs = ResultBuffers()
    pending = sorted(requests, key=lambda r: r.arrival_s)
    by_tag = {r.tag: r for r in requests}
    waiting: list[Request] = []
    t0 = time.perf_counter()
    active = 0
    active_sites = 0
    nxt = 0
    while nxt < len(pending) or waiting or active:
        now = time.perf_counter() - t0
        while nxt < len(pending) and (not realtime or pending[nxt].arrival_s <= now):
            waiting.append(pending[nxt])
            nxt += 1
        if policy == "sjf":
            waiting.sort(key=lambda r: (r.sites * r.nsteps, r.arrival_s))
        still = []
        for q, req in enumerate(waiting):
            if active and active_sites + req.sites > max_active_sites:
                still.extend(waiting[q:])  # the head of the order waits for room
                break
            p = req.params
            out = bufs.get((p.nz, p.ny, p.nx), _storage_dtype(p))
            if pool.submit_ic(p, device_ic(req), req.nsteps, req.tag, out=out):
                active += 1
                active_sites += req.sites
            else:
                bufs.put(out)
                rep.rejected_admissions += 1
                still.extend(waiting[q:])
                break
        waiting = still
        if active == 0:
            time.sleep(0.002)
            continue
        rep.max_active = max(rep.max_active, active)
        active = pool.step(chunk)
        done_t = time.perf_counter() - t0
        for r in pool.poll():
            req = by_tag[r.tag]
            rep.latencies_s[r.tag] = done_t - req.arrival_s
            rep.site_updates += req.sites * r.steps
            active_sites -= req.sites
            if on_result:
                on_result(req, r)
            bufs.put(r.psi)  # the state has been delivered; the buffer serves the next request
    rep.wall_s = time.perf_counter() - t0
    pool.close()
    return rep


def serve_one_at_a_time(requests: list[Request], realtime: bool = True) -> ServeReport:
    """Baseline: the plain one-solve-at-a-time FP64 path -- each request runs
    alone through the single-solve handle (complex128 storage), in arrival
    order, starting when it has arrived and the previous one has finished."""
    from .solver import Solver

    rep = ServeReport()
    bufs = ResultBuffers()
    t0 = time.perf_counter()
    for req in sorted(requests, key=lambda r: r.arrival_s):
        if realtime:
            wait = req.arrival_s - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        s = Solver(req.params.replace(storage="c128", compute="auto"))
        s.set_ic(device_ic(req))
        s.solver(req.nsteps)
        out = bufs.get(s.shape, np.complex128)
        s.get_state(out=out)  # the result is delivered, as in the batched loop
        bufs.put(out)
        s.close()
        rep.latencies_s[req.tag] = time.perf_counter() - t0 - req.arrival_s
        rep.site_updates += req.sites * req.nsteps
        rep.max_active = 1
    rep.wall_s = time.perf_counter() - t0
    return rep
