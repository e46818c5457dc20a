"""Tile-shape autotuner: pick the number of z planes per CTA work item
(tile_zc) that gives the fastest RK4 step, by timing candidates on the GPU,
either per (grid size, FD order, storage) in a pool of copies of one solve
(best_zc) or for a given batch of uneven solves as a whole (tune_mix: one
cap on the z-chunk length for all of them).  Results are cached in a JSON
file so a size or a mix is measured once per machine.

The x-y tile is fixed by the TMA box (32 x 8 sites); tile_zc trades the
z-halo re-read (2R planes per item) against the number of items, which
matters most for the small and uneven grids of a batched workload.  Shapes
are timed in that setting: a pool holding enough copies of the solve to
fill the GPU.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

from .solver import RunParams

CACHE = Path(os.environ.get("GPE_TUNE_CACHE", Path(__file__).resolve().parent / "tune_cache.json"))
CANDIDATES = (4, 8, 16, 32, 64)


def _key(n: int, order: int, storage: str) -> str:
    return f"n{n}_o{order}_{storage}"


def load_cache() -> dict:
    try:
        return json.loads(CACHE.read_text())
    except Exception:
        return {}


def save_cache(c: dict) -> None:
    CACHE.write_text(json.dumps(c, indent=1, sort_keys=True) + "\n")


def time_rk4(rp: RunParams, steps: int = 20, target_sites: int = 32 << 20) -> float:
    """Seconds per site per RK4 step when the GPU is kept busy with copies of
    this solve in one pool (the batched setting the tuned shape is used in).
    The copies add up to target_sites for every size, so small grids are
    timed on a saturated GPU as they run in a mixed batch, not on a
    half-empty one where many short items win."""
    import time

    from .pool import Pool

    n_sites = rp.nx * rp.ny * rp.nz
    copies = max(1, -(-target_sites // n_sites))
    pool = Pool(Pool.solve_bytes(rp) * copies + (64 << 20))
    psi = np.ones((rp.nz, rp.ny, rp.nx), np.complex64 if rp.storage == "c64" else np.complex128)
    for c in range(copies):
        pool.submit(rp, psi, steps + 4, c)
    pool.step(3)  # joins the batch, captures the step graph
    t0 = time.perf_counter()
    pool.step(steps)
    t = time.perf_counter() - t0
    pool.run_all()
    pool.close()
    return t / (steps * copies * n_sites)


def best_zc(n: int, order: int, storage: str, cache: dict | None = None) -> int:
    """Tuned tile_zc for a cubic n^3 grid (measures on a cache miss)."""
    own = cache is None
    cache = load_cache() if cache is None else cache
    k = _key(n, order, storage)
    if k not in cache:
        h = 0.25 * (n - 1)
        base = RunParams(nx=n, ny=n, nz=n, xr=h, yr=h, zr=h, tau=0.01, scheme="rk4", eqn_to_solve=4, bcs=1,
                         order=order, storage=storage)
        times = {zc: time_rk4(base.replace(tile_zc=zc)) for zc in CANDIDATES if zc <= n}
        cache[k] = {"zc": min(times, key=times.get), "s_per_site_step": times}
        if own:
            save_cache(cache)
    return int(cache[k]["zc"])


def tune(sizes, orders=(2, 4), storages=("c64",)) -> dict:
    cache = load_cache()
    for n in sizes:
        for o in orders:
            for st in storages:
                best_zc(n, o, st, cache)
    save_cache(cache)
    return cache


MIX_CAPS = (32, 48, 64, 96)


def _mix_key(params) -> str:
    import hashlib

    sig = sorted((p.nx, p.ny, p.nz, p.order, p.bcs, p.storage, p.scheme) for p in params)
    return "mix_" + hashlib.sha1(repr(sig).encode()).hexdigest()[:16]


def time_mix(params, states, cap: int, steps: int = 20) -> float:
    """Seconds per RK4 step of the whole batch with tile_zc = min(cap, nz)."""
    import time

    from .pool import Pool

    runs = [p.replace(tile_zc=min(cap, p.nz)) for p in params]
    pool = Pool(sum(Pool.solve_bytes(p) for p in runs) + (256 << 20))
    for k, (p, psi) in enumerate(zip(runs, states)):
        assert pool.submit(p, psi, steps + 4, k)
    pool.step(3)  # joins the batch, captures the step graph
    t0 = time.perf_counter()
    pool.step(steps)
    t = time.perf_counter() - t0
    pool.run_all()
    pool.close()
    return t / steps


def tune_mix(params, states, cache: dict | None = None) -> int:
    """The z-chunk cap that steps this batch of solves fastest (measured on a
    cache miss): each solve then uses tile_zc = min(cap, nz).  A cap suits
    an uneven batch better than per-size choices timed in homogeneous pools:
    the other solves keep the GPU busy, so items can be long."""
    own = cache is None
    cache = load_cache() if cache is None else cache
    k = _mix_key(params)
    if k not in cache:
        times = {cap: time_mix(params, states, cap) for cap in MIX_CAPS}
        cache[k] = {"cap": min(times, key=times.get), "s_per_step": times}
        if own:
            save_cache(cache)
    return int(cache[k]["cap"])
