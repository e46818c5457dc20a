"""Device initial conditions (gpe_set_ic, gpe_pool_submit_ic) against the
host restatement of src/ic.f90 (gpe_b200.ic) and the seeded random-phase
spectrum computed with numpy."""
from __future__ import annotations

import numpy as np
import pytest

from gpe_b200 import ic
from gpe_b200.pool import Pool
from gpe_b200.solver import RunParams, Solver

pytestmark = pytest.mark.gpu

RP = RunParams(nx=36, ny=30, nz=26, xr=8.75, yr=7.25, zr=6.25, scal=1.1, mu=6.0, g=1.3, omx=0.2, omy=0.15,
               omz=0.1, bcs=2, order=4)
RING = dict(plane="xz", x0=0.3, y0=-0.2, z0=0.1, r0=3.0, amp=0.2, mm=2, r1=0.3, kk=3, dir=-1.0)
LINE = dict(x0=0.3, y0=-0.4, z0=0.1, amp1=0.2, amp2=0.1, ll=3.0, sgn=-1.0, dir="z")
PULSE = dict(x0=0.4, y0=-0.3, z0=0.2, r0=2.5)


def host(kind):
    if kind == "ring":
        return ic.vortex_ring(RP, **RING)
    if kind == "line":
        return ic.vortex_line(RP, **LINE)
    if kind == "line_pade":
        return ic.vortex_line_pade(RP, **LINE)
    if kind == "fermi*line":
        return ic.fermi(RP) * ic.vortex_line(RP, **LINE)
    if kind == "ring*line":
        return ic.vortex_ring(RP, **RING) * ic.vortex_line(RP, **LINE)
    one = {"pade_pulse": lambda: ic.pade_pulse_ring(RP, "pulse", **PULSE),
           "pade_ring": lambda: ic.pade_pulse_ring(RP, "ring", **PULSE),
           "vortex_pair": lambda: ic.vortex_pair(RP), "sphere": lambda: ic.sphere(RP),
           "sphere2": lambda: ic.sphere2(RP), "wall": lambda: ic.wall(RP), "fermi": lambda: ic.fermi(RP)}
    out = None
    for f in kind.split("*"):
        v = one[f]()
        out = v if out is None else out * v
    return out


@pytest.mark.parametrize("kind", ["ring", "line", "line_pade", "fermi*line", "ring*line", "pade_pulse",
                                  "pade_ring", "vortex_pair", "sphere", "sphere2", "wall",
                                  "fermi*pade_pulse*vortex_pair"])
def test_closed_form_ics(gpu, kind):
    spec = ic.device_spec(*kind.split("*"), ring=RING, line=LINE, pulse=PULSE)
    s = Solver(RP)
    s.set_ic(spec)
    ref = host(kind)
    np.testing.assert_allclose(s.get_state(), ref, rtol=0, atol=1e-13 * max(1.0, float(np.abs(ref).max())))


def test_wall_ic_edge_and_complex64(gpu):
    # wall() switches at z = -30 (src/ic.f90:688-709): a grid with nodes on
    # both sides; and the Pade pulse in complex64 storage (FP64 per site,
    # one rounding to FP32)
    rp = RunParams(nx=16, ny=12, nz=41, xr=7.5, yr=5.5, zr=40.0, bcs=1, order=2)
    s = Solver(rp)
    s.set_ic(ic.device_spec("wall"))
    np.testing.assert_array_equal(s.get_state(), ic.wall(rp))
    s.close()
    s = Solver(RP.replace(storage="c64"))
    s.set_ic(ic.device_spec("pade_pulse", pulse=PULSE))
    ref = ic.pade_pulse_ring(RP, "pulse", **PULSE).astype(np.complex64)
    np.testing.assert_allclose(s.get_state(), ref, rtol=0, atol=1.2e-7 * float(np.abs(ref).max()))


@pytest.mark.parametrize("shape", [(32, 32, 32), (36, 30, 26)])
def test_random_phase_ic(gpu, shape):
    nx, ny, nz = shape
    rp = RunParams(nx=nx, ny=ny, nz=nz, xr=0.25 * (nx - 1), yr=0.25 * (ny - 1), zr=0.25 * (nz - 1), bcs=1, order=4)
    s = Solver(rp)
    s.set_ic(ic.device_spec("random_phase", seed=77, kc=1.4))
    dev = s.get_state()
    ref = ic.random_phase(rp, seed=77, kc=1.4)
    assert np.linalg.norm(dev - ref) / np.linalg.norm(ref) <= 1e-12
    assert np.mean(np.abs(dev) ** 2) == pytest.approx(1.0, rel=1e-12)


def test_pool_submit_ic_matches_host_state(gpu):
    rp = RP.replace(scheme="rk4")
    spec = ic.device_spec("fermi", "line", line=LINE)
    pool = Pool(2 * Pool.solve_bytes(rp) + (32 << 20))
    assert pool.submit_ic(rp, spec, 6, tag=1)
    assert pool.submit(rp, host("fermi*line"), 6, tag=2)
    res = {r.tag: r for r in pool.run_all()}
    np.testing.assert_allclose(res[1].psi, res[2].psi, rtol=0, atol=1e-12)
