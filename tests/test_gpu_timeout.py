"""The stage kernels' bounded waits: when a wait runs out the kernel records
it in the device status word, lets the copies it issued land and returns;
the host reports GPE_ERR_TIMEOUT and the handle or pool stays usable (the
reference's convention for such a failure is emergency_stop,
src/error.f90:24-46, which a host applies to the error code).

The expiry is made safely: gpe_test_expire_waits arms the status word so
that each work item waits, with a short limit, on a barrier that nothing
arrives at.  No kernel faults, traps or hangs.
"""
from __future__ import annotations

import numpy as np
import pytest

from gpe_b200 import _lib as L
from gpe_b200 import ic
from gpe_b200.solver import RunParams, Solver
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def ring_params(**kw):
    base = dict(nx=40, ny=36, nz=34, xr=9.75, yr=8.75, zr=8.25, tau=0.01, scheme="rk4", eqn_to_solve=4,
                bcs=2, order=4, g=1.0, mu=1.0)
    base.update(kw)
    return RunParams(**base)


@pytest.mark.parametrize("scheme", ["rk4", "rk45"])
@pytest.mark.parametrize("storage", ["c128", "c64"])
def test_expired_wait_reports_timeout_and_handle_recovers(gpu, scheme, storage):
    rp = ring_params(scheme=scheme, storage=storage, compute="f64" if storage == "c64" else "auto")
    psi0 = ic.vortex_ring(rp, "xy", r0=3.0)
    s = Solver(rp)
    s.set_state(psi0)
    assert s.lib.gpe_test_expire_waits(s.h) == L.GPE_OK
    with pytest.raises(L.GpeError) as e:
        s.solver(4)
    assert e.value.code == L.GPE_ERR_TIMEOUT
    assert "bounded wait" in str(e.value)
    # the same handle: the state after a timeout is unspecified, so set it
    # again; stepping then proceeds normally
    assert s.t == 0.0 and s.p == 0
    s.set_state(psi0)
    s.solver(6)
    out = s.get_state()
    # exactly what a fresh handle computes
    f = Solver(rp)
    f.set_state(psi0)
    f.solver(6)
    np.testing.assert_array_equal(out, f.get_state())
    assert (s.t, s.dt) == (f.t, f.dt)
    f.close()
    if storage == "c128":
        ref = Oracle(rp).run(psi0, 6)
        assert rel_l2(out, ref) <= (1e-10 if scheme == "rk45" else 1e-12)
    s.close()


def test_expired_wait_in_pool_retires_solves_and_pool_recovers(gpu):
    from gpe_b200.pool import Pool

    rps = [ring_params(), ring_params(scheme="rk45", nx=32, ny=30, nz=28, xr=7.75, yr=7.25, zr=6.75)]
    psis = [ic.vortex_ring(rp, "xy", r0=2.5) for rp in rps]
    pool = Pool(sum(Pool.solve_bytes(rp) for rp in rps) * 2 + (64 << 20))
    for k, (rp, psi) in enumerate(zip(rps, psis)):
        assert pool.submit(rp, psi, 8, k)
    assert pool.lib.gpe_pool_test_expire_waits(pool.h) == L.GPE_OK
    with pytest.raises(L.GpeError) as e:
        pool.step(8)
    assert e.value.code == L.GPE_ERR_TIMEOUT
    res = pool.poll()
    assert sorted(r.tag for r in res) == [0, 1]
    assert all(r.status == L.GPE_ERR_TIMEOUT for r in res)
    # the pool takes new work and runs it normally
    for k, (rp, psi) in enumerate(zip(rps, psis)):
        assert pool.submit(rp, psi, 8, 10 + k)
    res = {r.tag: r for r in pool.run_all()}
    assert sorted(res) == [10, 11]
    for k, (rp, psi) in enumerate(zip(rps, psis)):
        r = res[10 + k]
        assert r.status == L.GPE_OK and r.steps == 8
        ref = Oracle(rp).run(psi, 8)
        assert rel_l2(r.psi, ref) <= (1e-10 if rp.scheme == "rk45" else 1e-12)
    pool.close()
