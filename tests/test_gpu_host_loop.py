"""The C++ host driver's time loop against the same loop written out over
the CPU oracle (src/gpe.f90:136-280): the imaginary-time phase with
renormalisation, the switch to real time when successive norms agree to
1e-12 (src/gpe.f90:251-273), vortex-line imprinting in imaginary time
(imprint_vl, src/variables.f90:1166-1180), the restart products
(saved_restart / multiply_ic_restart, src/ic.f90:117-191), and the norm
records of real-time runs that the driver steps in chunks.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from gpe_b200.build import HOST
from gpe_b200.solver import RunParams
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def write_inputs(d: Path, *, nx, xr, tau, end_time, real_time, renorm=False, imprint_vl=False, restart=False,
                 saved_restart=False, multiply_ic_restart=False, save_rate=10, save_filter=False, om=1.0, mu=3.0,
                 ic="fermi()", scheme="rk4", order=2, bcs=2):
    d.mkdir(parents=True, exist_ok=True)
    L = lambda b: ".true." if b else ".false."  # noqa: E731
    (d / "run.in").write_text(f"""&run_params
  tau = {tau}, end_time = {end_time}, xr = {xr}, yr = {xr}, zr = {xr}
  scheme = '{scheme}', eqn_to_solve = 4, bcs = {bcs}, order = {order}
  restart = {L(restart)}, saved_restart = {L(saved_restart)}, multiply_ic_restart = {L(multiply_ic_restart)}
  renorm = {L(renorm)}, imprint_vl = {L(imprint_vl)}, stop_imag = .false., real_time = {L(real_time)}
/
&eqn_params
  Urhs = 0.0, diss_amp = 0.0, scal = 1.0, nv = 0.75, enerv = 0.75
  g = 1.0, mu = {mu}, nn = 2.0
  omx = {om}, omy = {om}, omz = {om}
/
&io_params
  save_rate = {save_rate}, save_rate2 = 1e9, save_rate3 = 1e9, p_save = 1e9
  save_3d = .false., save_filter = {L(save_filter)}, filter_kc = 6.0
/
&misc_params
  nbins = 256
/
""")
    (d / "parameters.in").write_text(f"""  integer, parameter :: pr = selected_real_kind(15,307)
  integer, parameter :: nx = {nx}
  integer, parameter :: ny = {nx}
  integer, parameter :: nz = {nx}
  type (line_param), parameter :: &
    vl1 = line_param(0.3_pr, -0.2_pr, 0.0_pr, &
      0.0_pr, 0.0_pr, 0.0_pr, 1.0_pr, 'z', .false.)
  type (ring_param), parameter :: &
    vr1 = ring_param('xy', 0.0_pr, 0.0_pr, 0.0_pr, 2.0_pr, &
      0.0_pr, 0, 0.0_pr, 0, 1.0_pr)
""")
    (d / "ic.in").write_text(f"  init_cond = {ic}\n")


def run(d):
    r = subprocess.run([str(HOST), "--dir", str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def read_end_state(path: Path):
    b = path.read_bytes()
    nx, ny, nz, p = np.frombuffer(b[:16], dtype=np.int32)
    t, im_t, dr, di = np.frombuffer(b[16:48], dtype=np.float64)
    psi = np.frombuffer(b[48:48 + 16 * nx * ny * nz], dtype=np.complex128).reshape(nz, ny, nx)
    return int(p), t, im_t, complex(dr, di), psi


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def params(nx, xr, tau, om=1.0, mu=3.0, real_time=True):
    return RunParams(nx=nx, ny=nx, nz=nx, xr=xr, yr=xr, zr=xr, tau=tau, scheme="rk4", eqn_to_solve=4, bcs=2,
                     order=2, g=1.0, mu=mu, nn=2.0, omx=om, omy=om, omz=om, real_time=real_time)


def oracle_loop(rp_imag, psi, end_time, renorm, imprint=None):
    """src/gpe.f90:136-280 for eqn 4 starting in imaginary time, written out
    over the oracle: returns (psi, t, im_t, p, switch step or None)."""
    o_im, o_re = Oracle(rp_imag), Oracle(rp_imag.replace(real_time=True))
    tau = rp_imag.tau
    real_time, t, im_t, p, dt, switched = False, 0.0, 0.0, 0, complex(0.0, -tau), None
    prev = o_im.get_norm(psi)  # src/gpe.f90:110-115
    if renorm:
        psi = o_im.renormalise(psi, prev)
    while t + im_t <= end_time:
        o = o_re if real_time else o_im
        psi = o.run(psi, 1)
        t, im_t = t + dt.real, im_t + abs(dt.imag)
        norm = o.get_norm(psi)
        relnorm = abs((norm - prev) / prev)
        if not real_time:
            if relnorm < 1e-12:
                real_time, im_t, switched = True, 0.0, p
                dt = complex(abs(dt.imag), abs(dt.real))
            if renorm:
                psi = o.renormalise(psi, norm)
            if imprint is not None:
                psi = np.abs(psi) * imprint
        prev = norm
        p += 1
    return psi, t, im_t, p, switched


def test_imaginary_time_converges_and_switches_to_real_time(gpu, tmp_path):
    nx, xr, tau, end_time = 20, 4.75, 0.02, 30.0
    d = tmp_path / "run"
    write_inputs(d, nx=nx, xr=xr, tau=tau, end_time=end_time, real_time=False, renorm=True)
    r = run(d)
    assert "Switching to real time" in r.stdout
    p, t, im_t, dt, psi = read_end_state(d / "proc0000" / "end_state.dat")
    rp = params(nx, xr, tau, real_time=False)
    o = Oracle(rp)
    ref, rt, rim, rpp, sw = oracle_loop(rp, o.fermi(), end_time, renorm=True)
    assert sw is not None and 0 < sw < rpp
    assert p == rpp and t == rt and im_t == rim and dt == complex(tau, 0.0)
    assert rel_l2(psi, ref) <= 1e-12


def test_imprint_vortex_line_in_imaginary_time(gpu, tmp_path):
    nx, xr, tau, end_time = 22, 5.25, 0.01, 0.3  # ends inside the imaginary phase
    d = tmp_path / "run"
    write_inputs(d, nx=nx, xr=xr, tau=tau, end_time=end_time, real_time=False, renorm=True, imprint_vl=True,
                 ic="fermi() * vortex_line(vl1)")
    run(d)
    p, t, im_t, dt, psi = read_end_state(d / "proc0000" / "end_state.dat")
    rp = params(nx, xr, tau, real_time=False)
    o = Oracle(rp)
    line = o.vortex_line(x0=0.3, y0=-0.2, dir="z")
    ref, rt, rim, rpp, sw = oracle_loop(rp, o.fermi() * line, end_time, renorm=True, imprint=line)
    assert sw is None and p == rpp and im_t == rim
    assert rel_l2(psi, ref) <= 1e-12
    # the imprinted phase is the line's: psi / |psi| = line / |line| where psi != 0
    m = np.abs(psi) > 1e-3
    assert np.allclose(psi[m] / np.abs(psi[m]), (line / np.abs(line))[m], atol=1e-12)


def test_restart_products_saved_filtered_and_ic(gpu, tmp_path):
    """saved_restart multiplies the end state by the saved filtered state
    (read as the reference's reader reads end_state_filtered.dat) and
    multiply_ic_restart by the ic.in product."""
    nx, xr, tau = 16, 3.75, 0.01
    d = tmp_path / "run"
    write_inputs(d, nx=nx, xr=xr, tau=tau, end_time=0.045, real_time=True, save_filter=True, ic="fermi()")
    run(d)
    p0, t0, im0, dt0, psi0 = read_end_state(d / "proc0000" / "end_state.dat")
    fb = (d / "proc0000" / "end_state_filtered.dat").read_bytes()
    n = nx ** 3
    assert len(fb) == 16 + 16 + 16 + 16 * n
    # the reader skips 4 integers and 2 reals, then takes n complex values
    f2 = np.frombuffer(fb[16 + 16:16 + 16 + 16 * n], dtype=np.complex128).reshape(nx, nx, nx)
    (d / "end_state0000.dat").write_bytes((d / "proc0000" / "end_state.dat").read_bytes())
    write_inputs(d, nx=nx, xr=xr, tau=tau, end_time=0.0, real_time=True, restart=True, saved_restart=True,
                 multiply_ic_restart=True, ic="vortex_ring(vr1)")
    run(d)  # end_time below t: no steps, the restart state is written back
    p1, t1, _, _, psi1 = read_end_state(d / "proc0000" / "end_state.dat")
    assert (p1, t1) == (p0, t0)
    ring = Oracle(params(nx, xr, tau)).vortex_ring("xy", r0=2.0)
    ref = (psi0 * f2) * ring
    assert rel_l2(psi1, ref) <= 1e-13


def test_chunked_real_time_norm_records(gpu, tmp_path):
    """Real-time fixed-step runs are stepped in chunks; the norm records
    (t, im_t, norm, relnorm at the save steps, relnorm against the previous
    step's norm) are those of stepping one step at a time."""
    from gpe_b200 import ic
    from gpe_b200.solver import Solver

    nx, xr, tau, end_time, save_rate = 24, 5.75, 0.01, 1.0, 7
    d = tmp_path / "run"
    write_inputs(d, nx=nx, xr=xr, tau=tau, end_time=end_time, real_time=True, save_rate=save_rate,
                 ic="fermi() * vortex_line(vl1)", order=4, bcs=1)
    run(d)
    recs = [[float(v) for v in line.split()] for line in (d / "norm.dat").read_text().splitlines()]
    rp = params(nx, xr, tau).replace(order=4, bcs=1)
    s = Solver(rp)
    s.set_ic(ic.device_spec("fermi", "line", line=dict(x0=0.3, y0=-0.2)))  # the driver's device IC
    want, prev, t = [], 1.0, 0.0
    while t <= end_time:
        info = s.solver(1, want_norm=True)
        t = s.t
        adt = abs(s.dt)
        b = adt * save_rate
        if t - np.floor(t / b) * b < adt:  # modulo(t+im_t, |dt| save_rate) < |dt|
            want.append([t, 0.0, info.norm, abs((info.norm - prev) / prev)])
        prev = info.norm
    assert len(recs) == len(want) and len(recs) > 10
    for got, w in zip(recs, want):
        assert got[0] == pytest.approx(w[0], rel=1e-8)
        assert got[2] == pytest.approx(w[2], rel=1e-8)
        assert got[3] == pytest.approx(w[3], rel=1e-6, abs=1e-17)
    p, tt, _, _, psi = read_end_state(d / "proc0000" / "end_state.dat")
    assert p == s.p and tt == s.t
    np.testing.assert_array_equal(psi, s.get_state())
