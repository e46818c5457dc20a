"""End-to-end runs of the C++ host driver on the GPU: the reference's input
files in, the reference's output files out, state identical to the same
solve through the Python interface and within 1e-12 of the CPU oracle;
restart from end_state continues the run exactly."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from gpe_b200 import ic
from gpe_b200.build import HOST
from gpe_b200.solver import RunParams, Solver
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

INPUTS = Path(__file__).resolve().parent / "golden" / "inputs"
RP = RunParams(nx=64, ny=64, nz=64, xr=15.75, yr=15.75, zr=15.75, tau=0.01, scheme="rk4", eqn_to_solve=4, bcs=2,
               order=2, g=1.0, mu=1.0)


def read_end_state(path: Path):
    b = path.read_bytes()
    nx, ny, nz, p = np.frombuffer(b[:16], dtype=np.int32)
    t, im_t, dr, di = np.frombuffer(b[16:48], dtype=np.float64)
    psi = np.frombuffer(b[48:], dtype=np.complex128).reshape(nz, ny, nx)
    return int(p), t, im_t, complex(dr, di), psi


def run(d):
    r = subprocess.run([str(HOST), "--dir", str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def test_host_run_and_restart(gpu, tmp_path):
    d = tmp_path / "run"
    shutil.copytree(INPUTS / "ring64", d)
    run(d)
    p, t, im_t, dt, psi = read_end_state(d / "proc0000" / "end_state.dat")
    assert p == 10 and t == pytest.approx(0.1, rel=1e-12) and im_t == 0.0 and dt == 0.01
    assert not (d / "RUNNING").exists() and not (d / "ERROR").exists()
    # same solve through the Python interface, device ring IC
    s = Solver(RP)
    s.set_ic(ic.device_spec("ring", ring=dict(plane="xy", r0=4.0)))
    s.solver(10)
    np.testing.assert_array_equal(psi, s.get_state())
    # the CPU oracle from the host ring IC
    ref = Oracle(RP).run(ic.vortex_ring(RP, "xy", r0=4.0), 10)
    assert np.linalg.norm(psi - ref) / np.linalg.norm(ref) <= 1e-12
    # time series: e17.9 records, energy every save_rate = 2 steps
    e = (d / "energy.dat").read_text().splitlines()
    nrm = (d / "norm.dat").read_text().splitlines()
    # (how many records depends on the accumulated t, as in the reference's
    # modulo(t+im_t, |dt|*save_rate) < |dt| test)
    assert len(e) >= 2 and all(len(x) == 51 for x in e)
    assert len(nrm) >= 2 and all(len(x) == 68 for x in nrm)
    # records are written at the steps where the save test fires; the norm
    # is conserved to O(dt^4) in real time
    assert all(float(x.split()[2]) == pytest.approx(s.get_norm(), rel=1e-5) for x in nrm)
    # restart from the end state for 10 more steps == 20 steps straight
    shutil.copy(d / "proc0000" / "end_state.dat", d / "end_state0000.dat")
    t_in = (d / "run.in").read_text().replace("restart             = .false.", "restart             = .true.")
    (d / "run.in").write_text(t_in.replace("end_time            = 0.095", "end_time            = 0.195"))
    run(d)
    p2, t2, _, _, psi2 = read_end_state(d / "proc0000" / "end_state.dat")
    s.solver(10)
    assert p2 == 20
    np.testing.assert_array_equal(psi2, s.get_state())


def test_host_pade_pulse_run(gpu, tmp_path):
    # an ic.in that asks for a Pade rarefaction pulse times the vortex pair
    # (src/ic.f90:518-636): the host builds it on the device; the end state
    # equals the Python interface's solve from the same device IC, and the
    # CPU oracle from the host restatement of the IC
    d = tmp_path / "run"
    shutil.copytree(INPUTS / "ring64", d)
    (d / "ic.in").write_text("  init_cond = pade_pulse_ring('pulse', 1.5_pr, -0.5_pr, 0.5_pr, 0.0_pr) * vortex_pair()\n")
    run(d)
    p, t, _, _, psi = read_end_state(d / "proc0000" / "end_state.dat")
    assert p == 10
    pulse = dict(x0=1.5, y0=-0.5, z0=0.5, r0=0.0)
    s = Solver(RP)
    s.set_ic(ic.device_spec("pade_pulse", "vortex_pair", pulse=pulse))
    s.solver(10)
    np.testing.assert_array_equal(psi, s.get_state())
    psi0 = ic.pade_pulse_ring(RP, "pulse", **pulse) * ic.vortex_pair(RP)
    ref = Oracle(RP).run(psi0, 10)
    assert np.linalg.norm(psi - ref) / np.linalg.norm(ref) <= 1e-12


def test_host_rejects_existing_end_state(gpu, tmp_path):
    d = tmp_path / "run"
    shutil.copytree(INPUTS / "ring64", d)
    (d / "end_state0000.dat").write_bytes(b"\0" * 64)
    r = subprocess.run([str(HOST), "--dir", str(d)], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "restart=.false. but end_state0000.dat exists" in (d / "ERROR").read_text()


def test_host_diagnostics_outputs(gpu, tmp_path):
    """mass.dat (condensed_particles), spectrum/idf/eta_time (spectrum),
    filtered<p>.dat (filtered_surface), psi_time.dat (save_time) and
    dens<p>.dat with the reference's itos file numbering."""
    from oracle import fft_diag as D

    d = tmp_path / "run"
    shutil.copytree(INPUTS / "ring64", d)
    t_in = (d / "run.in").read_text()
    t_in = t_in.replace("save_rate3    = 100.0", "save_rate3    = 0.05")
    t_in = t_in.replace("save_3d       = .false.",
                        "save_3d       = .true.\n  save_spectrum = .true.\n  save_filter   = .true.\n"
                        "  filter_kc     = 8.0")
    (d / "run.in").write_text(t_in)
    run(d)
    mass = (d / "mass.dat").read_text().splitlines()
    # at start (gpe.f90:116), first loop pass (t >= 0) and t >= 0.05; e17.9
    # records keep 9 significant digits (relative rounding up to 5e-9)
    assert len(mass) >= 3 and all(len(x) == 9 * 17 for x in mass)
    psi0 = ic.vortex_ring(RP, "xy", r0=4.0)
    rec, a = D.condensed_particles(psi0, RP.xr, RP.yr, RP.zr)
    first = [float(v) for v in mass[0].split()]
    V = RP.nx * RP.ny * RP.nz
    expect = [0.0, 0.0, rec["mass_density"], rec["n0"] / V, rec["M"], rec["n0"], rec["temp"], rec["temp2"],
              rec["H"] / V]
    for got, want in zip(first, expect):
        assert got == pytest.approx(want, rel=6e-9, abs=1e-300)
    spec = (d / "spectrum" / "spectrum0000000.dat").read_text().splitlines()
    eta, nharm, F = D.spectrum(a)
    assert len(spec) == 7 and all(len(x) == 35 for x in spec)
    for m, line in enumerate(spec):
        assert int(line[:9]) == m + 1 and int(line[9:18]) == nharm[m]
        # the device IC equals the host IC to ~1e-13, which is not small
        # relative to the near-empty high shells: absolute scale for those
        assert float(line[18:]) == pytest.approx(eta[m], rel=6e-9, abs=1e-11 * np.max(eta))
    idf = (d / "idf" / "idf0000000.dat").read_text().splitlines()
    assert len(idf) == RP.nx // 2
    assert [float(x[9:]) for x in idf] == pytest.approx(list(F), rel=6e-9, abs=1e-11 * F[-1])
    eta_t = (d / "eta_time.dat").read_text().splitlines()
    assert len(eta_t) == len(mass) and all(len(x) == 4 * 17 for x in eta_t)
    # filtered_surface stream file of the initial state
    b = (d / "proc0000" / "filtered0000000.dat").read_bytes()
    n = V
    assert len(b) == 8 + 9 * 4 + 16 * n + 8 * (RP.nx + RP.ny + RP.nz)
    filt = np.frombuffer(b[44:44 + 16 * n], dtype=np.complex128).reshape(RP.nz, RP.ny, RP.nx)
    ref = D.filtered_surface(a, 1.0, 8.0)
    assert np.linalg.norm(filt - ref) / np.linalg.norm(ref) <= 1e-12
    assert (d / "proc0000" / "dens0000000.dat").exists()
    pt = (d / "psi_time.dat").read_text().splitlines()
    assert len(pt) >= 2 and all(len(x) == 6 * 17 for x in pt)
    c = psi0[RP.nz // 2, RP.ny // 2, RP.nx // 2]
    v = [float(x) for x in pt[0].split()]
    assert v[2] == pytest.approx(c.real, rel=1e-8, abs=1e-12)
    assert v[3] == pytest.approx(c.imag, rel=1e-8, abs=1e-12)
    assert v[4] == pytest.approx(abs(c) ** 2, rel=1e-8, abs=1e-12)
    assert v[5] == pytest.approx(np.arctan2(c.imag + 1e-6, c.real), rel=1e-8, abs=1e-12)


def test_host_async_snapshots_hold_the_state_of_their_step(gpu, tmp_path):
    """dens<p>.dat files are written by a background thread from device
    snapshots while the time loop continues: each must hold the state of
    step p exactly."""
    d = tmp_path / "run"
    shutil.copytree(INPUTS / "ring64", d)
    t_in = (d / "run.in").read_text()
    t_in = t_in.replace("save_rate2    = 100.0", "save_rate2    = 0.03")
    t_in = t_in.replace("save_3d       = .false.", "save_3d       = .true.")
    (d / "run.in").write_text(t_in)
    run(d)
    saved = [int(x) for x in (d / "p_saved.dat").read_text().split()]
    assert 3 in saved and 6 in saved and 10 in saved
    s = Solver(RP)
    s.set_ic(ic.device_spec("ring", ring=dict(plane="xy", r0=4.0)))
    done = 0
    n = RP.nx * RP.ny * RP.nz
    for p in sorted(set(saved)):
        s.solver(p - done)
        done = p
        b = (d / "proc0000" / f"dens{p:07d}.dat").read_bytes()
        psi = np.frombuffer(b[8 + 36:8 + 36 + 16 * n], dtype=np.complex128).reshape(RP.nz, RP.ny, RP.nx)
        np.testing.assert_array_equal(psi, s.get_state())
