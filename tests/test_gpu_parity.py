"""Parity of the sm_100a stepper (through the C ABI) with the CPU oracle.

Tolerances: FP64 storage <= 1e-12 relative L2 (the target the reference's
plain FP64 method must meet); FP32 storage <= 1e-5 relative L2 and 1e-7
relative norm drift against the FP64 oracle where stated.
"""
from __future__ import annotations

import numpy as np
import pytest

from gpe_b200 import _lib as L
from gpe_b200 import ic
from gpe_b200.solver import RunParams, Solver
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def run_both(rp, psi0, steps, **kw):
    o = Oracle(rp)
    ref = o.run(psi0, steps)
    s = Solver(rp)
    s.set_state(psi0)
    info = s.solver(steps, **kw)
    out = s.get_state()
    return o, ref, s, out, info


def c1_params(**kw):
    # 64^3 ring, reflective, 2nd order, RK4 dt = 0.01, V = 0, mu = 1 (g = 1);
    # node-inclusive grid with dx = 0.5 (x_i = -15.75 + 0.5 i)
    base = dict(nx=64, ny=64, nz=64, xr=15.75, yr=15.75, zr=15.75, tau=0.01, scheme="rk4",
                eqn_to_solve=4, bcs=2, order=2, g=1.0, mu=1.0)
    base.update(kw)
    return RunParams(**base)


def test_c1_ring_rk4_1000_steps(gpu):
    rp = c1_params()
    psi0 = ic.vortex_ring(rp, "xy", r0=4.0)
    o, ref, s, out, info = run_both(rp, psi0, 1000, want_norm=True)
    assert rel_l2(out, ref) <= TOL64
    assert info.norm == pytest.approx(o.get_norm(ref), rel=TOL64)
    assert s.energy() == pytest.approx(o.energy(ref), rel=TOL64)
    assert s.t == o.clock.t and s.im_t == o.clock.im_t and s.p == 1000


def test_c1_eqn1_second_parity_case(gpu):
    rp = c1_params(eqn_to_solve=1)
    psi0 = ic.vortex_ring(rp, "xy", r0=4.0)
    o, ref, s, out, info = run_both(rp, psi0, 200)
    assert rel_l2(out, ref) <= TOL64


def golden_cases():
    from tests.golden.make_golden import CASES
    return [c[0] for c in CASES]


@pytest.mark.parametrize("name", golden_cases())
def test_golden_fixtures(gpu, name):
    from pathlib import Path

    from tests.golden.make_golden import CASES, SHAPE

    z = np.load(Path(__file__).resolve().parent / "golden" / "oracle_small.npz")
    kw = dict(next(c[1] for c in CASES if c[0] == name))
    rp = RunParams(**SHAPE, **kw)
    s = Solver(rp)
    s.set_state(z[f"{name}/psi0"])
    info = s.solver(int(z[f"{name}/steps"]), want_norm=True)
    out = s.get_state()
    # Adaptive RKF45 steps: the error estimate err = sum(dc_i K_i) cancels to
    # ~1e-6 of K, so rounding perturbs errmax (and hence the next dt) at the
    # ~1e-9 relative level in any two implementations; the trajectories then
    # agree to ~1e-11, not to rounding.  The first step (same dt) is exact
    # to rounding: see test_rk45_first_step_matches_to_rounding.
    tol = 1e-10 if kw.get("scheme") == "rk45" else TOL64
    assert rel_l2(out, z[f"{name}/psi"]) <= tol
    assert info.norm == pytest.approx(float(z[f"{name}/norm"]), rel=tol)
    assert s.energy() == pytest.approx(float(z[f"{name}/energy"]), rel=tol)
    clk = z[f"{name}/clock"]
    ttol = 1e-8 if kw.get("scheme") == "rk45" else 1e-12
    assert s.t == pytest.approx(clk[0], rel=ttol, abs=1e-300)
    assert s.im_t == pytest.approx(clk[1], rel=ttol, abs=1e-300)
    if kw.get("scheme") == "rk45":
        assert (s.dt.real, s.dt.imag) == pytest.approx((clk[2], clk[3]), rel=1e-8)


def test_rk45_first_step_matches_to_rounding(gpu):
    rp = RunParams(nx=26, ny=24, nz=30, xr=4.0, yr=4.0, zr=5.0, tau=0.01, scheme="rk45", eqn_to_solve=4,
                   bcs=2, order=4, g=1.0, mu=10.0, omx=0.05, omy=0.05, omz=0.025, gamma=0.05)
    psi0 = ic.fermi(rp) * ic.vortex_line_pade(rp, dir="z")
    o, ref, s, out, info = run_both(rp, psi0, 1)
    assert rel_l2(out, ref) <= 1e-13
    assert info.errmax == pytest.approx(o.clock.errmax, rel=1e-7)
    assert s.dt.real == pytest.approx(o.clock.dt_re, rel=1e-8)


SIZES = [(17, 13, 11), (33, 20, 9), (40, 7, 12)]


@pytest.mark.parametrize("shape", SIZES)
@pytest.mark.parametrize("eqn", [1, 2, 3, 4])
@pytest.mark.parametrize("bcs", [1, 2])
@pytest.mark.parametrize("order", [2, 4])
def test_matrix_rk4(gpu, shape, eqn, bcs, order):
    nx, ny, nz = shape
    rp = RunParams(nx=nx, ny=ny, nz=nz, xr=4.0, yr=3.0, zr=2.0, tau=0.003, scheme="rk4", eqn_to_solve=eqn,
                   bcs=bcs, order=order, g=1.3, mu=0.7, omx=0.2, omy=0.3, omz=0.1,
                   Urhs=0.2 if eqn != 4 else 0.0, diss_amp=0.1 if eqn in (1, 3) else 0.0)
    rng = np.random.default_rng(nx * 100 + eqn * 10 + bcs + order)
    psi0 = (rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx))) * 0.3 + 1.0
    o, ref, s, out, info = run_both(rp, psi0, 4)
    assert rel_l2(out, ref) <= TOL64


@pytest.mark.parametrize("scheme", ["euler", "rk2", "rk4", "rk45"])
@pytest.mark.parametrize("real_time", [True, False])
def test_schemes_real_and_imaginary_time(gpu, scheme, real_time):
    # For RKF45 the condensate must fill the box: where psi = 0 the error
    # ratio |err|/(|psi| + dt|f| + 1e-30) is rounding noise over ~0 and the
    # adaptive dt is then not reproducible between any two implementations.
    trap = dict(mu=10.0, omx=0.05, omy=0.05, omz=0.025) if scheme == "rk45" else dict(mu=2.0, omx=0.3, omy=0.3,
                                                                                       omz=0.2)
    rp = RunParams(nx=24, ny=22, nz=20, xr=5.0, yr=5.0, zr=5.0, tau=0.004, scheme=scheme, eqn_to_solve=4,
                   bcs=2, order=4, g=1.0, real_time=real_time, **trap)
    psi0 = ic.fermi(rp) * ic.vortex_line_pade(rp, dir="z")
    o, ref, s, out, info = run_both(rp, psi0, 8)
    tol = 1e-10 if scheme == "rk45" else TOL64  # see test_golden_fixtures
    assert rel_l2(out, ref) <= tol
    assert s.t == pytest.approx(o.clock.t, rel=1e-9, abs=1e-300)
    assert s.im_t == pytest.approx(o.clock.im_t, rel=1e-9, abs=1e-300)


def test_rk45_step_control_sequence(gpu):
    # large initial tau forces rejections; dt sequence must follow the oracle
    rp = RunParams(nx=24, ny=20, nz=28, xr=4.0, yr=4.0, zr=5.0, tau=0.2, scheme="rk45", eqn_to_solve=4,
                   bcs=2, order=4, g=1.0, mu=10.0, omx=0.05, omy=0.05, omz=0.025, gamma=0.05)
    psi0 = ic.fermi(rp) * ic.vortex_line_pade(rp, dir="z")
    o = Oracle(rp)
    s = Solver(rp)
    s.set_state(psi0)
    psi = psi0
    for _ in range(6):
        psi = o.run(psi, 1)
        s.solver(1)
        assert s.dt.real == pytest.approx(o.clock.dt_re, rel=1e-8)
        assert s.t == pytest.approx(o.clock.t, rel=1e-9)
    assert rel_l2(s.get_state(), psi) <= 1e-10
    assert o.clock.rejected >= 1


def test_norm_energy_renormalise(gpu):
    rp = RunParams(nx=30, ny=26, nz=22, xr=5.0, yr=4.0, zr=3.0, bcs=1, order=4, nn=3.0)
    rng = np.random.default_rng(3)
    psi0 = rng.standard_normal((22, 26, 30)) + 1j * rng.standard_normal((22, 26, 30))
    o = Oracle(rp)
    s = Solver(rp)
    s.set_state(psi0)
    n = s.get_norm()
    assert n == pytest.approx(o.get_norm(psi0), rel=1e-13)
    assert s.energy() == pytest.approx(o.energy(psi0), rel=1e-12)
    s.renormalise(n)
    assert rel_l2(s.get_state(), o.renormalise(psi0, n)) <= 1e-15
    assert s.get_norm() == pytest.approx(3.0, rel=1e-13)


def test_fused_energy_equals_standalone(gpu):
    rp = c1_params(nx=40, ny=36, nz=32)
    psi0 = ic.vortex_ring(rp, "xy", r0=4.0)
    s = Solver(rp)
    s.set_state(psi0)
    e0 = s.energy()
    info = s.solver(3, want_energy=True, want_norm=True)
    assert info.energy == pytest.approx(e0, rel=1e-13)
    assert info.norm == pytest.approx(s.get_norm(), rel=1e-13)


def test_state_roundtrip_both_dtypes(gpu):
    rp = RunParams(nx=19, ny=17, nz=15, storage="c128")
    rng = np.random.default_rng(11)
    psi = rng.standard_normal((15, 17, 19)) + 1j * rng.standard_normal((15, 17, 19))
    s = Solver(rp)
    s.set_state(psi)
    np.testing.assert_array_equal(s.get_state(), psi)
    s.set_state(psi.astype(np.complex64))
    np.testing.assert_array_equal(s.get_state(np.complex64), psi.astype(np.complex64))


def test_nonfinite_is_reported(gpu):
    rp = RunParams(nx=16, ny=16, nz=16)
    psi = np.ones((16, 16, 16), np.complex128)
    psi[3, 4, 5] = np.nan
    s = Solver(rp)
    s.set_state(psi)
    with pytest.raises(L.GpeError) as e:
        s.solver(1, want_norm=True)
    assert e.value.code == L.GPE_ERR_NONFINITE


@pytest.mark.parametrize("compute", ["f32", "f64"])
def test_fp32_storage_vs_fp64_oracle(gpu, compute):
    rp = c1_params(nx=48, ny=48, nz=48, xr=11.75, yr=11.75, zr=11.75, bcs=1, order=4, eqn_to_solve=2,
                   tau=0.005)
    psi0 = ic.random_phase(rp, seed=5, kc=1.5)
    o = Oracle(rp)
    ref = o.run(psi0, 200)
    s = Solver(rp.replace(storage="c64", compute=compute))
    s.set_state(psi0)
    info = s.solver(200, want_norm=True)
    out = s.get_state()
    err = rel_l2(out, ref)
    drift = abs(info.norm - o.get_norm(ref)) / o.get_norm(ref)
    print(f"fp32 storage ({compute} compute): rel_l2={err:.3e} norm drift={drift:.3e}")
    assert err <= 1e-5
    assert drift <= 1e-7


def test_fp32_storage_trapped_vs_fp64_oracle(gpu):
    # eqn 4 with a trap: the FP32 stencil forms V from float halves
    rp = c1_params(nx=40, ny=40, nz=40, xr=9.75, yr=9.75, zr=9.75, bcs=2, order=4, eqn_to_solve=4,
                   tau=0.005, mu=5.0, omx=0.1, omy=0.1, omz=0.15)
    psi0 = ic.fermi(rp) * ic.vortex_line_pade(rp, dir="z")
    o = Oracle(rp)
    ref = o.run(psi0, 200)
    s = Solver(rp.replace(storage="c64", compute="f32"))
    s.set_state(psi0)
    info = s.solver(200, want_norm=True)
    err = rel_l2(s.get_state(), ref)
    drift = abs(info.norm - o.get_norm(ref)) / o.get_norm(ref)
    print(f"fp32 storage, trapped: rel_l2={err:.3e} norm drift={drift:.3e}")
    assert err <= 1e-5
    assert drift <= 1e-7


C2_RP = RunParams(nx=256, ny=256, nz=256, xr=63.75, yr=63.75, zr=63.75, tau=0.005, scheme="rk4",
                  eqn_to_solve=2, bcs=1, order=4)


@pytest.fixture(scope="module")
def c2_oracle_200():
    """The roofline workload (256^3 random phase, periodic, 4th order, RK4
    dt = 0.005, eqn 2) run 200 steps by the FP64 CPU oracle, once for the
    tests of this module: (psi0, psi_200, norm, energy)."""
    psi0 = ic.random_phase(C2_RP, seed=1234, kc=1.5)
    o = Oracle(C2_RP)
    ref = o.run(psi0, 200)
    return psi0, ref, o.get_norm(ref), o.energy(ref)


@pytest.mark.slow
def test_fp32_storage_c2_256_cubed_vs_oracle(gpu, c2_oracle_200):
    """The roofline workload in complex64 storage with the FP32 stencil, 200
    steps, against the FP64 CPU oracle on the same initial state."""
    psi0, ref, nref, eref = c2_oracle_200
    s = Solver(C2_RP.replace(storage="c64", compute="f32"))
    s.set_state(psi0)
    s.solver(200)
    out = s.get_state()
    n32, e32 = s.get_norm(), s.energy()
    s.close()
    err = rel_l2(out, ref)
    drift = abs(n32 - nref) / nref
    edrift = abs(e32 - eref) / abs(eref)
    print(f"fp32 storage 256^3, 200 steps: rel_l2={err:.3e} norm drift={drift:.3e} energy drift={edrift:.3e}")
    assert err <= 1e-5
    assert drift <= 1e-7


def test_fp32_storage_rk45_trapped_vs_fp64_oracle(gpu):
    """The trapped RKF45 workload on a smaller grid (48 x 48 x 96, dx = 0.25,
    reflective, 4th order, eqn 4 with gamma = 0.05, mu = 10, trap (0.05,
    0.05, 0.025), TF x Pade vortex line, eps = 1e-6): complex64 storage with
    FP64 step control, 200 accepted steps, against the FP64 oracle's RKF45.
    The two runs choose their own step sizes, so they end at slightly
    different times; the oracle is advanced to the FP32 run's final time
    (its last RKF45 step that stays below it, then one FP64 RK4 step of the
    remaining interval) and compared there."""
    rp = RunParams(nx=48, ny=48, nz=96, xr=5.875, yr=5.875, zr=11.875, tau=0.01, scheme="rk45",
                   eqn_to_solve=4, bcs=2, order=4, g=1.0, mu=10.0, omx=0.05, omy=0.05, omz=0.025, gamma=0.05)
    psi0 = ic.fermi(rp) * ic.vortex_line_pade(rp, dir="z")
    s = Solver(rp.replace(storage="c64", compute="f32"))
    s.set_state(psi0)
    info = s.solver(200)
    out = s.get_state()
    t32, acc32, rej32 = s.t, 200, info.rejected
    n32 = s.get_norm()
    s.close()
    o = Oracle(rp)
    psi, acc64 = psi0, 0
    while True:
        t_before = o.clock.t
        nxt = o.run(psi, 1)
        if o.clock.t > t32:
            break
        psi, acc64 = nxt, acc64 + 1
    gap = t32 - t_before
    assert 0.0 <= gap < 0.05
    ref = Oracle(rp.replace(scheme="rk4", tau=gap)).run(psi, 1) if gap > 0 else psi
    nref = o.get_norm(ref)
    err = rel_l2(out, ref)
    drift = abs(n32 - nref) / nref
    print(f"fp32 storage RKF45 trapped: rel_l2={err:.3e} norm drift={drift:.3e} t={t32:.6f} "
          f"accepted/rejected fp32 {acc32}/{rej32}, fp64 oracle {acc64}/{o.clock.rejected} (to t={t_before:.6f})")
    # the step sizes differ (FP32 storage perturbs the error estimate), not
    # the rate at which the controller advances
    assert abs(acc64 - acc32) <= 0.1 * acc32
    assert err <= 1e-5
    assert drift <= 1e-7


@pytest.mark.slow
def test_c2_256_cubed_periodic_o4(gpu, c2_oracle_200):
    """The roofline workload in complex128, 200 steps through the replayed
    step graph, against the FP64 CPU oracle: psi, norm and energy."""
    psi0, ref, nref, eref = c2_oracle_200
    s = Solver(C2_RP)
    s.set_state(psi0)
    info = s.solver(200, want_norm=True)
    out = s.get_state()
    e = s.energy()
    s.close()
    assert rel_l2(out, ref) <= TOL64
    assert info.norm == pytest.approx(nref, rel=TOL64)
    assert e == pytest.approx(eref, rel=TOL64)


def test_snapshot_while_stepping(gpu):
    """gpe_snapshot_begin captures the state of its point in the stream even
    when stepping continues before gpe_snapshot_wait."""
    rp = c1_params(nx=40, ny=36, nz=32, xr=9.75, yr=8.75, zr=7.75)
    psi0 = ic.vortex_ring(rp, "xy", r0=3.0)
    s = Solver(rp)
    s.set_state(psi0)
    s.solver(5)
    at5 = s.get_state()
    s.snapshot_begin()
    s.solver(7, wait=False)
    snap = s.snapshot_wait()
    np.testing.assert_array_equal(snap, at5)
    s.snapshot_begin(np.complex64)
    s.sync()
    at12 = s.get_state()
    np.testing.assert_array_equal(s.snapshot_wait(), at12.astype(np.complex64))
    s.close()


@pytest.mark.parametrize("shape", [(6, 6, 6), (7, 6, 9), (33, 6, 7)])
@pytest.mark.parametrize("order,bcs", [(2, 1), (2, 2), (4, 1), (4, 2)])
@pytest.mark.parametrize("scheme", ["euler", "rk4", "rk45"])
def test_smallest_grids_match_oracle(gpu, shape, order, bcs, scheme):
    """The smallest admitted grids (6 points per axis): every site sits next
    to a ghost face, tiles are mostly empty, and a z-chunk holds the whole
    axis; (33, 6, 7) also puts one site in a second x tile."""
    nx, ny, nz = shape
    rp = RunParams(nx=nx, ny=ny, nz=nz, xr=0.5 * (nx - 1), yr=0.5 * (ny - 1), zr=0.5 * (nz - 1), tau=0.005,
                   scheme=scheme, eqn_to_solve=4, bcs=bcs, order=order, g=1.0, mu=2.0, omx=0.3, omy=0.2, omz=0.25)
    rng = np.random.default_rng(nx * 100 + ny * 10 + nz + order + bcs)
    psi0 = 1.0 + 0.2 * (rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx)))
    o, ref, s, out, info = run_both(rp, psi0, 12, want_norm=True)
    tol = 1e-10 if scheme == "rk45" else TOL64
    assert rel_l2(out, ref) <= tol
    assert info.norm == pytest.approx(o.get_norm(ref), rel=tol)
    s.close()


def test_grid_below_the_minimum_is_rejected(gpu):
    rp = RunParams(nx=5, ny=8, nz=8, xr=2.0, yr=3.5, zr=3.5)
    with pytest.raises(L.GpeError) as e:
        Solver(rp)
    assert e.value.code == L.GPE_ERR_BADARG


def test_async_state_copies_pipeline(gpu):
    """gpe_set_state_async / gpe_get_state_async in a pipeline of three
    solves from different inputs: each result equals the synchronous path's,
    although transfers overlap the neighbouring solves' steps."""
    rp = c1_params(nx=40, ny=36, nz=34, xr=9.75, yr=8.75, zr=8.25)
    ins = [L.pinned_empty((34, 36, 40), np.complex128) for _ in range(3)]
    outs = [L.pinned_empty((34, 36, 40), np.complex128) for _ in range(3)]
    for q, a in enumerate(ins):
        a[...] = ic.vortex_ring(rp, "xy", r0=2.0 + q)
    ref = []
    s = Solver(rp)
    for a in ins:
        s.set_state(a)
        s.solver(6)
        ref.append(s.get_state())
    for a, o in zip(ins, outs):
        s.set_state_async(a)
        s.solver(6, wait=False)
        s.get_state_async(o)
    s.sync()
    for o, r in zip(outs, ref):
        np.testing.assert_array_equal(o, r)
    s.close()
