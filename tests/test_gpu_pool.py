"""Batched solves (gpe_pool_*): every solve evolves exactly as it would
alone -- bitwise -- whether it runs by itself in a pool, mixed with solves of
other sizes, boundary conditions, orders, precisions and schemes, or through
the single-solve handle; admission respects the HBM budget."""
from __future__ import annotations

import numpy as np
import pytest

from gpe_b200 import ic
from gpe_b200.pool import Pool
from gpe_b200.solver import RunParams, Solver
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def params(n, bcs, order, scheme="rk4", storage="c128", eqn=4, **kw):
    nx, ny, nz = n
    base = dict(nx=nx, ny=ny, nz=nz, xr=0.25 * (nx - 1), yr=0.25 * (ny - 1), zr=0.25 * (nz - 1), tau=0.01,
                scheme=scheme, eqn_to_solve=eqn, bcs=bcs, order=order, g=1.0, mu=1.0, storage=storage)
    if scheme == "rk45":
        base.update(mu=10.0, omx=0.05, omy=0.05, omz=0.05, gamma=0.05)
    base.update(kw)
    return RunParams(**base)


def state(rp, seed):
    if rp.scheme == "rk45":
        psi = ic.fermi(rp) * ic.vortex_line_pade(rp, dir="z")
    elif seed % 2:
        psi = ic.random_phase(rp, seed=seed, kc=1.5)
    else:
        psi = ic.vortex_ring(rp, "xy", r0=2.0 + seed % 3)
    return psi.astype(np.complex64) if rp.storage == "c64" else psi


MIX = [
    ((32, 32, 32), 1, 4, "rk4", "c128"),
    ((48, 40, 36), 2, 2, "rk4", "c128"),
    ((33, 17, 20), 2, 4, "rk4", "c64"),
    ((64, 48, 40), 1, 2, "rk4", "c64"),
    ((40, 36, 30), 2, 4, "rk45", "c128"),
    ((30, 28, 26), 2, 4, "rk45", "c64"),
]


def run_alone_handle(rp, psi0, steps):
    s = Solver(rp)
    s.set_state(psi0)
    s.solver(steps)
    out = s.get_state(np.complex64 if rp.storage == "c64" else np.complex128)
    return out, s


def test_pool_mix_equals_alone_bitwise(gpu):
    steps = 12
    cases = [(params(*c[:3], scheme=c[3], storage=c[4]), i) for i, c in enumerate(MIX)]
    budget = sum(Pool.solve_bytes(rp) for rp, _ in cases) + (64 << 20)
    mixed = Pool(budget)
    for rp, i in cases:
        assert mixed.submit(rp, state(rp, i), steps, tag=i)
    res = {r.tag: r for r in mixed.run_all(max_steps=5)}
    assert sorted(res) == list(range(len(cases)))
    for rp, i in cases:
        r = res[i]
        assert r.status == 0 and r.steps == steps
        # alone in a pool
        alone = Pool(Pool.solve_bytes(rp) + (16 << 20))
        assert alone.submit(rp, state(rp, i), steps, tag=99)
        (ra,) = alone.run_all(max_steps=5)
        np.testing.assert_array_equal(r.psi, ra.psi)
        assert r.norm == ra.norm and r.t == ra.t and r.dt == ra.dt
        # the single-solve handle
        out, s = run_alone_handle(rp, state(rp, i), steps)
        np.testing.assert_array_equal(r.psi, out)
        assert r.t == s.t and r.im_t == s.im_t
        # the pool's norm is that of the final state (formed on a chunk's last step only)
        assert r.norm == pytest.approx(s.get_norm(), rel=1e-12)
        if rp.scheme == "rk45":
            assert r.dt == s.dt
        # and directly against the FP64 CPU oracle on the same initial state
        # (not RKF45 with complex64 storage: its step sizes differ from the
        # FP64 oracle's, so equal step counts are different times; that case
        # is compared at matched times in test_gpu_parity.py)
        if not (rp.scheme == "rk45" and rp.storage == "c64"):
            o = Oracle(rp.replace(storage="c128"))
            oref = o.run(state(rp, i).astype(np.complex128), steps)
            err = np.linalg.norm(r.psi - oref) / np.linalg.norm(oref)
            if rp.storage == "c64":
                assert err <= 1e-5
            else:
                assert err <= (1e-10 if rp.scheme == "rk45" else 1e-12)


def test_pool_budget_admission(gpu):
    rp = params((48, 48, 48), 1, 4)
    need = Pool.solve_bytes(rp)
    pool = Pool(2 * need + need // 2)
    psi = state(rp, 1)
    assert pool.submit(rp, psi, 4, tag=1)
    assert pool.submit(rp, psi, 4, tag=2)
    assert not pool.submit(rp, psi, 4, tag=3)  # over budget: caller retries later
    res = pool.run_all()
    assert sorted(r.tag for r in res) == [1, 2]
    assert pool.free_bytes() >= 2 * need
    assert pool.submit(rp, psi, 4, tag=3)
    (r3,) = pool.run_all()
    np.testing.assert_array_equal(r3.psi, res[0].psi)


def test_pool_continuous_batching(gpu):
    # a solve submitted while others are mid-run joins at the next step and
    # still evolves exactly as alone
    rp1 = params((40, 40, 40), 2, 4)
    rp2 = params((36, 44, 28), 1, 2)
    pool = Pool(Pool.solve_bytes(rp1) + Pool.solve_bytes(rp2) + (32 << 20))
    assert pool.submit(rp1, state(rp1, 2), 20, tag=1)
    pool.step(6)
    assert pool.submit(rp2, state(rp2, 3), 10, tag=2)
    res = {r.tag: r for r in pool.run_all(max_steps=4)}
    for tag, rp, seed, n in ((1, rp1, 2, 20), (2, rp2, 3, 10)):
        out, _ = run_alone_handle(rp, state(rp, seed), n)
        np.testing.assert_array_equal(res[tag].psi, out)
    assert res[2].start_s >= res[2].submit_s


@pytest.mark.parametrize("storage, scheme", [("c64", "rk4"), ("c128", "rk4"), ("c64", "rk45"), ("c128", "rk45")])
def test_classes_beyond_the_parameter_space(gpu, storage, scheme):
    # a launch carries the stage arguments of up to 60 solves in its
    # parameter space; a class of 64 solves takes the device-table path.
    # Both give each solve's states bitwise as the single-solve handle
    # does (one class of 64 and one of 7 solves in the same pool).
    steps = 4 if scheme == "rk4" else 3
    rps = [params((8 + (k % 3), 8, 6 + (k % 2)), 1 + (k % 2), 4, scheme=scheme, storage=storage) for k in range(64)]
    rps += [params((10, 9, 8), 2, 2, scheme=scheme, storage=storage) for _ in range(7)]
    pool = Pool(sum(Pool.solve_bytes(rp) for rp in rps) + (64 << 20))
    psis = [state(rp, k) for k, rp in enumerate(rps)]
    for k, (rp, psi) in enumerate(zip(rps, psis)):
        assert pool.submit(rp, psi, steps, k)
    res = {r.tag: r for r in pool.run_all()}
    pool.close()
    for k in (0, 1, 2, 5, 33, 63, 64, 70):
        alone, s = run_alone_handle(rps[k], psis[k], steps)
        s.close()
        np.testing.assert_array_equal(res[k].psi, alone, err_msg=f"solve {k}")
