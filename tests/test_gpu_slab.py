"""z-slab decomposition of one solve (gpe_create_slab): slabs of an
in-process hub (one host thread per slab, one GPU) and the NCCL transport
(one rank on a periodic axis exchanging with itself) against the same solve
on the whole grid.  Per-site arithmetic is the same, so psi must agree bit
for bit; norms and energies are sums in another order (1e-13)."""
from __future__ import annotations

import numpy as np
import pytest

from gpe_b200 import _lib as L
from gpe_b200 import ic, slab
from gpe_b200.solver import RunParams, Solver
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def whole(rp, psi, nsteps):
    s = Solver(rp)
    s.set_state(psi)
    info = s.solver(nsteps, want_norm=True)
    out = s.get_state(), info.norm, (s.t, s.im_t, s.dt, s.p)
    s.close()
    return out


CASES = {
    "periodic_o4_rk4_eqn2": (RunParams(nx=32, ny=28, nz=30, xr=7.75, yr=6.75, zr=7.25, tau=0.01, scheme="rk4",
                                       eqn_to_solve=2, bcs=1, order=4), "random"),
    "reflective_o2_rk4_eqn4_trap": (RunParams(nx=30, ny=32, nz=27, xr=7.25, yr=7.75, zr=6.5, tau=0.01,
                                              scheme="rk4", eqn_to_solve=4, bcs=2, order=2, mu=3.0, omx=0.2,
                                              omy=0.3, omz=0.25), "ring"),
    "reflective_o4_rk2_eqn1_diss": (RunParams(nx=28, ny=28, nz=26, xr=6.75, yr=6.75, zr=6.25, tau=0.005,
                                              scheme="rk2", eqn_to_solve=1, bcs=2, order=4, diss_amp=0.3),
                                    "ring"),
    "periodic_o2_euler_eqn3": (RunParams(nx=32, ny=24, nz=24, xr=7.75, yr=5.75, zr=5.75, tau=0.002,
                                         scheme="euler", eqn_to_solve=3, bcs=1, order=2), "random"),
}


def initial(rp, kind):
    if kind == "random":
        return ic.random_phase(rp, seed=21, kc=1.5)
    return ic.vortex_ring(rp, "xy", r0=2.5)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("nslabs", [2, 3])
def test_hub_slabs_match_whole_grid(gpu, name, nslabs):
    rp, kind = CASES[name]
    psi = initial(rp, kind)
    ref, ref_norm, ref_t = whole(rp, psi, 12)
    out, norm, t = slab.step_decomposed(rp, psi, nslabs, 12)
    assert np.array_equal(out, ref)
    assert norm == pytest.approx(ref_norm, rel=1e-13)
    assert t == ref_t
    # and directly against the CPU oracle (the reference's single-rank path)
    o = Oracle(rp)
    oref = o.run(psi, 12)
    assert np.linalg.norm(out - oref) / np.linalg.norm(oref) <= 1e-12
    assert norm == pytest.approx(o.get_norm(oref), rel=1e-12)


@pytest.mark.parametrize("storage", ["c128", "c64"])
def test_hub_slabs_rk45_same_step_control(gpu, storage):
    rp = RunParams(nx=28, ny=30, nz=32, xr=6.75, yr=7.25, zr=7.75, tau=0.02, scheme="rk45", eqn_to_solve=4,
                   bcs=2, order=4, mu=4.0, omx=0.3, omy=0.25, omz=0.2, gamma=0.05, storage=storage)
    psi = ic.fermi(rp) * ic.vortex_line(rp, x0=0.3, y0=-0.2)
    ref, ref_norm, ref_t = whole(rp, psi, 8)
    out, norm, t = slab.step_decomposed(rp, psi, 3, 8)
    assert np.array_equal(out, ref)
    assert t == ref_t  # same t, im_t, dt and p: every slab took the same decisions
    assert norm == pytest.approx(ref_norm, rel=1e-13)
    # against the FP64 CPU oracle over the first step (the adaptive-step
    # tolerance: a rejected first attempt sets the accepted dt from an error
    # estimate that cancels to ~1e-6 of K)
    out1, _, _ = slab.step_decomposed(rp, psi, 3, 1)
    oref = Oracle(rp.replace(storage="c128")).run(psi, 1)
    err = np.linalg.norm(out1 - oref) / np.linalg.norm(oref)
    assert err <= (1e-10 if storage == "c128" else 1e-6)


def test_hub_energy_and_norm_calls(gpu):
    rp, kind = CASES["reflective_o2_rk4_eqn4_trap"]
    psi = initial(rp, kind)
    s = Solver(rp)
    s.set_state(psi)
    e_ref, n_ref = s.energy(), s.get_norm()
    s.close()

    def body(sl):
        sl.set_state(psi[sl.k0:sl.k0 + sl.nzl])
        return sl.energy(), sl.get_norm()

    res = slab.run_threaded(rp, 3, body)
    for e, n in res:
        assert e == pytest.approx(e_ref, rel=1e-13)
        assert n == pytest.approx(n_ref, rel=1e-13)


def test_nccl_single_rank_periodic_self_exchange(gpu):
    rp, kind = CASES["periodic_o4_rk4_eqn2"]
    psi = initial(rp, kind)
    ref, ref_norm, _ = whole(rp, psi, 10)
    s = Solver(rp, rank=0, nranks=1, nccl_id=slab.nccl_unique_id())
    s.set_state(psi)
    info = s.solver(10, want_norm=True)
    out = s.get_state()
    s.close()
    assert np.array_equal(out, ref)
    assert info.norm == pytest.approx(ref_norm, rel=1e-13)


def test_slab_argument_checks(gpu):
    rp, _ = CASES["periodic_o4_rk4_eqn2"]
    lib = L.load()
    import ctypes as C

    cp = rp.to_c()
    h = C.c_void_p()
    hub = slab.SlabHub(2)
    # 30 planes over 6 slabs leaves 5 per slab (< 6)
    assert lib.gpe_create_slab(C.byref(cp), 0, 6, None, None, C.byref(h)) == L.GPE_ERR_BADARG
    # exactly one transport
    assert lib.gpe_create_slab(C.byref(cp), 0, 2, None, None, C.byref(h)) == L.GPE_ERR_BADARG
    # the hub was made for 2 slabs
    assert lib.gpe_create_slab(C.byref(cp), 0, 3, None, hub.h, C.byref(h)) == L.GPE_ERR_BADARG
    hub.close()


def test_hub_detects_a_slab_that_never_calls_in(gpu, monkeypatch):
    """Failure detection on the host: slab 1 stops after creation; slab 0's
    next collective call returns GPE_ERR_TIMEOUT instead of hanging."""
    import threading

    monkeypatch.setenv("GPE_HUB_TIMEOUT_S", "2")
    rp, kind = CASES["periodic_o4_rk4_eqn2"]
    psi = initial(rp, kind)
    hub = slab.SlabHub(2)
    s0 = Solver(rp, rank=0, nranks=2, hub=hub)
    made = threading.Event()
    holder = {}

    def idle():
        holder["s1"] = Solver(rp, rank=1, nranks=2, hub=hub)
        made.set()

    t = threading.Thread(target=idle)
    t.start()
    made.wait(30)
    t.join()
    with pytest.raises(L.GpeError) as e:
        s0.set_state(psi[s0.k0:s0.k0 + s0.nzl])
    assert e.value.code == L.GPE_ERR_TIMEOUT or "timeout" in str(e.value)
    # the hub is broken now: the other slab fails at once as well
    s1 = holder["s1"]
    with pytest.raises(L.GpeError):
        s1.set_state(psi[s1.k0:s1.k0 + s1.nzl])
    s0.close()
    s1.close()
    hub.close()
