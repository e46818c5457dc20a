"""The serving loop (continuous batching of a request stream): every request
finishes, and each result is bitwise the state the same request reaches
alone through its own single-solve handle -- whatever else was in the batch
when it ran (RK4 and RKF45, FP64 and FP32 storage, device-built initial
states)."""
from __future__ import annotations

import numpy as np
import pytest

from gpe_b200.serve import device_ic, initial_state, make_requests, serve
from gpe_b200.solver import Solver
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def test_served_results_equal_single_handles(gpu):
    reqs = make_requests(8, rate_per_s=1000.0, seed=11, sizes=(24, 32, 40), steps=(5, 12))
    got = {}

    def keep(req, r):
        got[req.tag] = (r.status, r.steps, np.array(r.psi, copy=True))

    rep = serve(reqs, budget_bytes=1 << 30, chunk=4, realtime=False, on_result=keep)
    assert sorted(got) == sorted(r.tag for r in reqs)
    assert sorted(rep.latencies_s) == sorted(got)
    assert rep.site_updates == sum(r.sites * r.nsteps for r in reqs)
    kinds = {(r.params.scheme, r.params.storage) for r in reqs}
    assert len(kinds) >= 3  # the stream mixes schemes and precisions
    for req in reqs:
        status, steps, psi = got[req.tag]
        assert status == 0 and steps == req.nsteps
        s = Solver(req.params)
        s.set_ic(device_ic(req))
        s.solver(req.nsteps)
        alone = s.get_state(np.complex64 if req.params.storage == "c64" else np.complex128)
        s.close()
        np.testing.assert_array_equal(psi, alone)
        # and against the FP64 CPU oracle from the host restatement of the
        # request's initial state (not RKF45 with complex64 storage: its
        # step sizes differ from the FP64 oracle's, see test_gpu_parity.py)
        if req.params.scheme == "rk45" and req.params.storage == "c64":
            continue
        rp64 = req.params.replace(storage="c128")
        psi0 = initial_state(req.__class__(**{**req.__dict__, "params": rp64}))
        oref = Oracle(rp64).run(psi0, req.nsteps)
        err = np.linalg.norm(psi - oref) / np.linalg.norm(oref)
        if req.params.storage == "c64":
            assert err <= 1e-5
        else:
            assert err <= (1e-10 if req.params.scheme == "rk45" else 1e-12)
