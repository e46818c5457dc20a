"""Benchmark of the B200 Gross-Pitaevskii stepper.

Workload (N = 1 line): 256^3 grid, periodic BCs, 4th-order centred FD, RK4
dt = 0.005, eqn_to_solve = 2, seeded random-phase initial state, complex128
storage and FP64 arithmetic.  One bench "step" = CHUNK (200) RK4 time steps
of the whole grid.  Each field is 280 MB > L2 (126 MB), so no L2 flush is
needed between steps.

  value  site-updates/s with the state resident in HBM (CUDA events on the
         solver's stream, max over ranks, summed over ranks' sites)
  e2e    the same metric through the C ABI with host buffers: every bench
         step copies psi in from pinned host memory (gpe_set_state), runs
         CHUNK steps (gpe_step) and copies psi out (gpe_get_state)

Multi-GPU (torchrun): every rank advances its own independent solve (replicas,
weak scaling); there is no data-path collective.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "RK4 site-updates/s & HBM roofline %, 256^3; batched-solve p50/p99 latency"
UNIT = "site-updates/s"
CHUNK = 200
WORKLOAD = dict(nx=256, ny=256, nz=256, xr=63.75, yr=63.75, zr=63.75, tau=0.005, scheme="rk4",
                eqn_to_solve=2, bcs=1, order=4)
CONFIG = {"workload": "256^3 periodic, 4th-order FD, RK4 dt=0.005, eqn 2, random-phase IC (seed 1234, kc 1.5), "
                      "complex128", "grid": [256, 256, 256], "steps_per_bench_step": CHUNK,
          "l2_policy": "inputs larger than L2 (each field 280 MB)", "parallelism": "replicas"}


def measured_hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic_per_site(kind: str):
    """DRAM bytes per site of one stage launch from the committed ncu
    summary (profiles/), or None."""
    f = ROOT / "profiles" / "ncu_rk4_stage_256cubed.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(f"traffic_bytes_per_site[{kind}]"):
            try:
                return float(line.split("=")[1].split()[0])
            except Exception:
                return None
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline(steps: int = 2):
    """The reference's CPU path (C restatement in oracle/, OpenMP on all host
    cores, per-call diss/Vtrap rebuild as the reference does) on a bounded
    sample of the workload: `steps` RK4 steps of the 256^3 grid."""
    from gpe_b200 import ic
    from gpe_b200.solver import RunParams
    from oracle.pyoracle import Oracle, load

    lib = load()
    cores = os.cpu_count() or 1
    lib.or_set_threads(cores)
    rp = RunParams(**WORKLOAD)
    psi = ic.random_phase(rp, seed=1234, kc=1.5)
    o = Oracle(rp)
    o.faithful_cost(True)
    o.run(psi, 1)  # first-touch / warm-up
    t0 = time.perf_counter()
    o.run(psi, steps)
    dt = time.perf_counter() - t0
    n = rp.nx * rp.ny * rp.nz
    return {"value": n * steps / dt, "unit": UNIT, "cores": int(lib.or_get_threads()), "kind": "port",
            "sample": f"{steps} RK4 steps of the 256^3 workload (C restatement of solve.f90/derivs.f90, "
                      "reference binary unavailable: no Fortran compiler)"}


def run_reference(args, ws, rank):
    """--impl reference: the reference's CPU implementation (oracle port) on
    the host cores; rank 0 only."""
    if rank != 0:
        return 0
    from gpe_b200 import ic
    from gpe_b200.solver import RunParams
    from oracle.pyoracle import Oracle, load

    lib = load()
    cores = os.cpu_count() or 1
    lib.or_set_threads(cores)
    rp = RunParams(**WORKLOAD)
    psi = ic.random_phase(rp, seed=1234, kc=1.5)
    o = Oracle(rp)
    o.faithful_cost(True)
    per = 1  # RK4 steps per bench step (bounded sample)
    for _ in range(args.warmup):
        psi = o.run(psi, per)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        psi = o.run(psi, per)
    dt = time.perf_counter() - t0
    n = rp.nx * rp.ny * rp.nz
    v = n * per * args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG, steps_per_bench_step=per), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": int(lib.or_get_threads()), "kind": "port",
                             "sample": f"{per} RK4 step of the 256^3 workload per bench step; C restatement "
                                       "of solve.f90/derivs.f90 (reference binary unavailable: no Fortran compiler)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def read_profile(s):
    """Per-kind (total ms, launches, B/site) from the library's event timing."""
    import ctypes as C

    from gpe_b200 import _lib as L

    prof = {}
    for kind, name in enumerate(L.KIND_NAMES):
        tot, n, bps = C.c_double(), C.c_int64(), C.c_double()
        s.lib.gpe_profile_get(s.h, kind, C.byref(tot), C.byref(n), C.byref(bps))
        if n.value:
            prof[name] = (tot.value, n.value, bps.value)
    return prof


def fp32_storage_leg(args, torch, psi0):
    """The same 256^3 workload with complex64 storage (FP32 stencil, FP64
    stage combinations and reductions): device-resident site-updates/s."""
    from gpe_b200.solver import RunParams, Solver

    out = {}
    for compute in ("f32", "f64"):
        rp = RunParams(**WORKLOAD, storage="c64", compute=compute)
        s = Solver(rp)
        s.set_state(psi0)
        stream = torch.cuda.ExternalStream(s.stream())
        for _ in range(max(1, args.warmup)):
            s.solver(CHUNK, wait=False)
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n = max(1, args.steps // 2)
        e0.record(stream)
        for _ in range(n):
            s.solver(CHUNK, wait=False)
        e1.record(stream)
        s.sync()
        ms = e0.elapsed_time(e1)
        # per-kernel times from a second, event-instrumented pass
        s.lib.gpe_profile(s.h, 1)
        for _ in range(n):
            s.solver(CHUNK, wait=False)
        s.sync()
        prof = read_profile(s)
        s.close()
        n_sites = rp.nx * rp.ny * rp.nz
        step_bytes = sum(v[2] * v[1] for v in prof.values()) * n_sites
        step_ms = sum(v[0] for v in prof.values())
        out[compute + "_compute"] = {
            "value": n_sites * CHUNK * n / (ms * 1e-3), "unit": UNIT,
            "bytes_per_site_step": sum(v[2] * v[1] for v in prof.values()) / (CHUNK * n),
            "all_stage_kernels_gbs": step_bytes / (step_ms * 1e-3) / 1e9,
            "per_kind_gbs": {k: v[2] * n_sites / (v[0] / v[1] * 1e-3) / 1e9 for k, v in prof.items()},
            "per_kind_ms": {k: v[0] / v[1] for k, v in prof.items()}}
    return out


ACC_STEPS = 2000


def fp32_accuracy_leg(psi0, steps: int = ACC_STEPS):
    """Accuracy of complex64 storage at the full workload: the 256^3 random
    phase state advanced `steps` RK4 steps (dt = 0.005) with complex64
    storage, against the complex128 FP64 GPU path from the same initial
    state (that path matches the FP64 CPU oracle to <= 1e-12 relative L2 in
    the parity tests).  rel_l2 = |psi32 - psi64| / |psi64| over all sites;
    norm / energy drift = |X32 - X64| / |X64| at the final step (get_norm
    quadrature; energy() as the reference defines it)."""
    from gpe_b200.solver import RunParams, Solver

    def run(**kw):
        s = Solver(RunParams(**WORKLOAD, **kw))
        s.set_state(psi0)
        n0, e0 = s.get_norm(), s.energy()
        s.solver(steps)
        out = s.get_state()
        n1, e1 = s.get_norm(), s.energy()
        s.close()
        return out, n0, e0, n1, e1

    ref, n0, e0, nref, eref = run()
    den = float(np.linalg.norm(ref.ravel()))
    res = {"steps": steps, "reference": "complex128 FP64 GPU path from the same initial state (parity tests pin it "
                                        "to the FP64 CPU oracle at <= 1e-12 rel L2)",
           "fp64_self_norm_drift": abs(nref - n0) / n0, "fp64_self_energy_drift": abs(eref - e0) / abs(e0)}
    for compute in ("f32", "f64"):
        out, _, _, n1, e1 = run(storage="c64", compute=compute)
        res[compute + "_compute"] = {
            "rel_l2": float(np.linalg.norm((out - ref).ravel())) / den,
            "norm_drift": abs(n1 - nref) / nref,
            "energy_drift": abs(e1 - eref) / abs(eref)}
        del out
    return res


def rk45_leg(args, torch):
    """Trapped-condensate RKF45 workload: 192x192x384, dx = 0.25, reflective,
    4th order, eqn 4 with damping gamma = 0.05, mu = 10, trap (0.05, 0.05,
    0.025), TF x Pade vortex line, eps = 1e-6, complex128.  Site-updates/s
    count accepted steps; each attempt moves 576 B/site."""
    from gpe_b200 import ic
    from gpe_b200.solver import RunParams, Solver

    rp = RunParams(nx=192, ny=192, nz=384, xr=23.875, yr=23.875, zr=47.875, tau=0.01, scheme="rk45",
                   eqn_to_solve=4, bcs=2, order=4, g=1.0, mu=10.0, omx=0.05, omy=0.05, omz=0.025, gamma=0.05)
    psi0 = ic.fermi(rp) * ic.vortex_line_pade(rp, dir="z")
    s = Solver(rp)
    s.set_state(psi0)
    s.solver(10)  # settle the adaptive step
    s.lib.gpe_profile(s.h, 1)
    per = 20
    t0 = time.perf_counter()
    acc = rej = 0
    for _ in range(max(1, args.steps // 2)):
        info = s.solver(per)
        acc += info.accepted
        rej += info.rejected
    wall = time.perf_counter() - t0
    prof = read_profile(s)
    dev_ms = sum(v[0] for v in prof.values())
    attempts = acc + rej
    n_sites = rp.nx * rp.ny * rp.nz
    s.close()
    return {"value": n_sites * acc / wall, "unit": UNIT, "accepted": acc, "rejected": rej,
            "dt_last": abs(s.dt), "device_ms_per_attempt": dev_ms / attempts,
            "device_gbs": 576 * n_sites * attempts / (dev_ms * 1e-3) / 1e9,
            "timing": "wall clock around gpe_step (includes the 8-byte error-norm read-back per attempt)"}


C4_STEPS = 500
C4_SHORT = 200


def c4_mix(storage: str = "c64", tuned: bool = True):
    """The 64 uneven solves of the batched workload: cubic sizes uniform in
    {32, 48, ..., 160}, periodic/reflective and 2nd/4th order mixed (seeded),
    RK4 dt = 0.01, eqn 4, ring (r0 in [2,6]) / random-phase (cutoff in
    [1,2]) initial states alternating.  tuned: tile_zc = min(cap, n) with
    the z-chunk cap the autotuner picks for this batch (measured on a cache
    miss), else the pool's default.  Returns [(params, page-locked input,
    page-locked result buffer)] and the cache."""
    from gpe_b200 import _lib as L
    from gpe_b200 import autotune
    from gpe_b200 import ic
    from gpe_b200.solver import RunParams

    rng = np.random.default_rng(64)
    cache = autotune.load_cache() if tuned else {}
    dt = np.complex64 if storage == "c64" else np.complex128
    solves = []
    for k in range(64):
        n = int(rng.choice(np.arange(32, 161, 16)))
        bcs, order = int(rng.choice([1, 2])), int(rng.choice([2, 4]))
        r0, kc = float(rng.uniform(2, 6)), float(rng.uniform(1, 2))
        h = 0.25 * (n - 1)
        rp = RunParams(nx=n, ny=n, nz=n, xr=h, yr=h, zr=h, tau=0.01, scheme="rk4", eqn_to_solve=4, bcs=bcs,
                       order=order, g=1.0, mu=1.0, storage=storage)
        psi = ic.vortex_ring(rp, "xy", r0=r0) if k % 2 == 0 else ic.random_phase(rp, seed=k, kc=kc)
        # the caller's input and result buffers: page-locked, allocated once
        host = L.pinned_empty(psi.shape, dt)
        host[...] = psi
        solves.append((rp, host, L.pinned_empty(psi.shape, dt)))
    if tuned:
        cap = autotune.tune_mix([s[0] for s in solves], [s[1] for s in solves], cache)
        solves = [(rp.replace(tile_zc=min(cap, rp.nz)), a, b) for rp, a, b in solves]
        autotune.save_cache(cache)
    return solves, cache


def batched_leg(args, torch):
    """The c4_mix solves in one pool, complex64 storage with FP64
    reductions, 500 steps, the z-chunk cap from the autotuner.  Timed on the
    host clock from the first submission to the last retired result (state
    upload and download included); latencies are per solve, all submitted at
    t = 0."""
    from gpe_b200.pool import Pool

    solves, cache = c4_mix("c64", tuned=True)
    budget = sum(Pool.solve_bytes(rp) for rp, _, _ in solves) + (256 << 20)
    sites = sum(rp.nx * rp.ny * rp.nz for rp, _, _ in solves)

    def run(steps):
        pool = Pool(budget)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k, (rp, psi, out) in enumerate(solves):
            assert pool.submit(rp, psi, steps, k, out=out)
        res = pool.run_all(max_steps=steps)
        wall = time.perf_counter() - t0
        pool.close()
        return wall, res

    run(2)  # warm-up: autotuned shapes, graph capture paths, first-touch
    wall, res = run(C4_STEPS)
    lat = np.array([r.finish_s - r.submit_s for r in res])
    # the same mix resident on the device: time C4_SHORT steps of all solves
    pool = Pool(budget)
    for k, (rp, psi, out) in enumerate(solves):
        assert pool.submit(rp, psi, C4_SHORT + 20, k, out=out)
    pool.step(10)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pool.step(C4_SHORT)
    torch.cuda.synchronize()
    resident = time.perf_counter() - t0
    pool.run_all()
    pool.close()
    return {"value": sites * C4_STEPS / wall, "unit": UNIT, "solves": len(res), "sites": sites,
            "steps": C4_STEPS, "wall_s": wall, "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "storage": "c64",
            "stepping_rate": sites * C4_SHORT / resident,
            "tile_zc": {f"n{rp.nx}": rp.tile_zc for rp, _, _ in solves},
            "timing": "value: host clock, first submit to last result, uploads/downloads included (the caller's "
                      "states and result buffers in page-locked host memory); stepping_rate: host clock around "
                      f"{C4_SHORT} steps of the whole mix resident on the device (synchronised both sides)"}


def ncu_batch_case(args) -> int:
    """Profiling target for the batched kernel: the c4_mix solves (storage
    --storage, pool default z-chunks) submitted to one pool, 12 RK4 steps."""
    from gpe_b200.pool import Pool

    solves, _ = c4_mix(args.storage, tuned=False)
    pool = Pool(sum(Pool.solve_bytes(rp) for rp, _, _ in solves) + (256 << 20))
    for k, (rp, psi, out) in enumerate(solves):
        assert pool.submit(rp, psi, 12, k, out=out)
    pool.run_all()
    pool.close()
    return 0


SERVING_SEED = 2024


def serving_leg(n_requests: int, torch):
    """The serving workload's first n_requests requests (Poisson 20/s, seed
    2024; sizes 48^3..256^3; 200-5000 RK4/RKF45 steps; order 2/4; V = 0 or a
    trap; ring / line / random-phase initial states built on the device;
    FP64 or FP32 storage): continuous batching with shortest-job-first
    admission from one HBM budget, against the plain one-solve-at-a-time FP64
    path on the same requests.  Latency = completion - arrival (host clock)."""
    from gpe_b200 import serve

    reqs = serve.make_requests(n_requests, seed=SERVING_SEED)
    free, _ = torch.cuda.mem_get_info()
    budget = int(free * 0.85)
    batched = serve.serve(reqs, budget, chunk=50).summary()
    single = serve.serve_one_at_a_time(reqs).summary()
    work = sum(r.sites * r.nsteps for r in reqs)
    return {"requests": len(reqs), "seed": SERVING_SEED, "rate_per_s": 20.0,
            "offered_site_steps": work, "arrival_span_s": reqs[-1].arrival_s,
            "offered_site_steps_per_s": work / reqs[-1].arrival_s,
            "sustained_site_steps_per_s": batched["site_updates_per_s"],
            "policy": "shortest job first among arrived requests, <= 48 Mi sites in flight, HBM budget 85% of free",
            "continuous_batching": batched, "one_at_a_time_fp64": single,
            "throughput_ratio": batched["site_updates_per_s"] / single["site_updates_per_s"],
            "p50_ratio": batched["p50_s"] / single["p50_s"], "p99_ratio": batched["p99_s"] / single["p99_s"]}


def run_serving(args) -> int:
    """Serving sample: the first `--requests` requests of the synthetic
    stream (Poisson 20/s; sizes 48^3..256^3; 200-5000 RK4/RKF45 steps;
    order 2/4; V = 0 or a trap; ring / line / random-phase ICs; FP64 or FP32
    storage) served with continuous batching from one HBM budget, then the
    same requests through the plain one-solve-at-a-time FP64 path."""
    import torch

    from gpe_b200 import serve

    torch.cuda.set_device(0)
    reqs = serve.make_requests(args.requests)
    free, total = torch.cuda.mem_get_info()
    budget = int(free * 0.85)
    batched = serve.serve(reqs, budget, chunk=50).summary()
    single = serve.serve_one_at_a_time(reqs).summary()
    work = sum(r.sites * r.nsteps for r in reqs)
    line = {"metric": "serving p50/p99 latency and site-updates/s", "requests": len(reqs),
            "offered_site_steps": work, "arrival_span_s": reqs[-1].arrival_s,
            "offered_site_steps_per_s": work / reqs[-1].arrival_s, "budget_bytes": budget,
            "continuous_batching": batched, "one_at_a_time_fp64": single,
            "throughput_ratio": batched["site_updates_per_s"] / single["site_updates_per_s"]}
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="device-resident leg only (tuning sweeps)")
    ap.add_argument("--no-extras", action="store_true", help="skip the FP32-storage and RKF45 legs")
    ap.add_argument("--ncu-case", action="store_true",
                    help="profiling target: set up the workload and run 2 RK4 steps, nothing else")
    ap.add_argument("--serving", action="store_true",
                    help="serving workload: Poisson stream of mixed solves, continuous batching vs one at a time")
    ap.add_argument("--requests", type=int, default=40, help="--serving: requests in the sample")
    ap.add_argument("--serving-requests", type=int, default=200,
                    help="requests of the serving sample on the main line (0 = skip)")
    ap.add_argument("--storage", default="c128", choices=["c128", "c64"],
                    help="storage of the --ncu-case / --quick workload")
    ap.add_argument("--batch", action="store_true",
                    help="with --ncu-case: the 64 uneven solves of the batched workload in one pool "
                         "(pool default z-chunks), 12 RK4 steps")
    args = ap.parse_args()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    if args.serving:
        return run_serving(args)
    if args.ncu_case and args.batch:
        return ncu_batch_case(args)

    import torch

    from gpe_b200 import dist

    torch.cuda.set_device(local % max(1, torch.cuda.device_count()))
    pg = dist.init(backend=os.environ.get("GPE_DIST_BACKEND", "nccl"), timeout_s=120)

    from gpe_b200 import _lib as L
    from gpe_b200 import ic
    from gpe_b200.solver import RunParams, Solver

    rp = RunParams(**WORKLOAD)
    n_sites = rp.nx * rp.ny * rp.nz
    psi0 = ic.random_phase(rp, seed=1234, kc=1.5)
    if args.ncu_case or args.quick:
        rp = rp.replace(storage=args.storage, compute="f32" if args.storage == "c64" else "auto")
    s = Solver(rp)
    s.set_state(psi0)
    stream = torch.cuda.ExternalStream(s.stream())
    if args.ncu_case:
        s.solver(2)
        s.close()
        return 0

    def barrier():
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()

    max_over_ranks = dist.max_over_ranks

    # ---- device-resident throughput -------------------------------------
    for _ in range(args.warmup):
        s.solver(CHUNK, wait=False)
    s.sync()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            s.solver(CHUNK, wait=False)
        ev1.record(stream)
        s.sync()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = n_sites * CHUNK * args.steps * ws / (ms * 1e-3)
    gpu_launches = 4 * CHUNK * args.steps

    # per-kernel times for the roofline: a second timed region of the same
    # workload with CUDA events around every stage kernel (those events cost
    # a few percent, so the value above is timed without them)
    prof_steps = max(1, args.steps // 2)
    s.lib.gpe_profile(s.h, 1)
    for _ in range(prof_steps):
        s.solver(CHUNK, wait=False)
    s.sync()
    prof = read_profile(s)
    s.lib.gpe_profile(s.h, 0)

    # roofline of the dominant kernel: the stage kind with the largest share
    # of the step's device time
    dom = max(prof, key=lambda k: prof[k][0])
    tot, n, bps = prof[dom]
    avg_ms = tot / n
    achieved = bps * n_sites / (avg_ms * 1e-3) / 1e9
    peak, peak_src = measured_hbm_peak()
    traffic_ps = ncu_traffic_per_site(dom)
    step_bytes = sum(v[2] * v[1] for v in prof.values()) * n_sites
    step_ms = sum(v[0] for v in prof.values())
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (traffic_ps * n_sites) if traffic_ps else None,
                "kernel": f"k_stage_tma<double2,double,R=2,{dom.upper()}> (RK4 stage {dom[-1]})",
                "share": tot / sum(v[0] for v in prof.values()),
                "bytes_per_site": bps, "avg_launch_ms": avg_ms, "peak_source": peak_src,
                "timing": f"CUDA events around each stage kernel on the solver's stream over {prof_steps} bench "
                          "step(s) of the same workload right after the timed region",
                "frac_of_vendor_8000": achieved / 8000.0,
                "all_stage_kernels_gbs": step_bytes / (step_ms * 1e-3) / 1e9,
                "per_kind_ms": {k: v[0] / v[1] for k, v in prof.items()}}

    if args.quick:
        s.close()
        if rank == 0:
            print(json.dumps({"value": value, "unit": UNIT, "ms_per_step": ms / args.steps,
                              "zc": os.environ.get("GPE_ZC"), "roofline": roofline}), flush=True)
        return 0

    # ---- end to end through the C ABI with host buffers ------------------
    host_in = torch.empty((rp.nz, rp.ny, rp.nx), dtype=torch.complex128, pin_memory=True)
    host_in.numpy()[...] = psi0
    host_out = torch.empty_like(host_in, pin_memory=True)
    hin, hout = host_in.numpy(), host_out.numpy()
    # every bench step: the input state goes in from page-locked host memory,
    # CHUNK steps run, the result comes back; the transfers run on the
    # handle's copy stream (gpe_set_state_async / gpe_get_state_async) and
    # overlap the neighbouring bench steps' compute
    for _ in range(1):
        s.set_state_async(hin)
        s.solver(CHUNK, wait=False)
        s.get_state_async(hout)
    s.sync()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.set_state_async(hin)
        s.solver(CHUNK, wait=False)
        s.get_state_async(hout)
    s.wait_copies()  # the end event comes after the last result has landed
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    barrier()
    ems = max_over_ranks(e0.elapsed_time(e1))
    e2e = {"value": n_sites * CHUNK * args.steps * ws / (ems * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": int(hin.nbytes), "d2h_bytes_per_step": int(hout.nbytes),
           "ms_per_step": ems / args.steps,
           "path": "gpe_set_state_async -> gpe_step_async -> gpe_get_state_async per bench step, page-locked host "
                   "buffers, transfers on the copy stream overlapping compute"}
    gpu_launches += args.steps * (4 * CHUNK + 2)
    assert np.isfinite(hout).all(), "non-finite state"

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": CONFIG,
            "e2e": e2e, "roofline": roofline, "clocks": clk.summary(), "gpu_launches": gpu_launches}
    if not args.no_extras and ws == 1:  # the extra legs are single-GPU workloads
        line["fp32_storage"] = fp32_storage_leg(args, torch, psi0)
        line["fp32_storage"]["speedup_vs_fp64"] = line["fp32_storage"]["f32_compute"]["value"] / (value / ws)
        line["fp32_storage"]["accuracy"] = fp32_accuracy_leg(psi0)
        if args.serving_requests > 0:
            line["serving"] = serving_leg(args.serving_requests, torch)
        line["rk45_trapped"] = rk45_leg(args, torch)
        line["batched_c4"] = batched_leg(args, torch)
        line["batched_c4"]["speedup_vs_plain_fp64"] = line["batched_c4"]["value"] / (value / ws)
        line["batched_c4"]["stepping_speedup_vs_plain_fp64"] = line["batched_c4"]["stepping_rate"] / (value / ws)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    s.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        dist.finalize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
