"""The C++ host driver (gpe_b200/bin/gpe_host): parsing of the reference's
input files and its error convention, on CPU (no GPU needed)."""
from __future__ import annotations

import json
import shutil
import subprocess
from pathlib import Path

import pytest

from gpe_b200.build import HOST

INPUTS = Path(__file__).resolve().parent / "golden" / "inputs"


def run_host(d, *args):
    return subprocess.run([str(HOST), "--dir", str(d), *args], capture_output=True, text=True, timeout=60)


@pytest.fixture
def ring_dir(tmp_path):
    d = tmp_path / "ring64"
    shutil.copytree(INPUTS / "ring64", d)
    return d


def test_parse_reference_inputs(ring_dir):
    r = run_host(ring_dir, "--parse-only")
    assert r.returncode == 0, r.stderr
    p = json.loads(r.stdout)
    assert (p["nx"], p["ny"], p["nz"], p["pr"]) == (64, 64, 64, 8)
    assert p["scheme"] == 2 and p["eqn"] == 4 and p["bcs"] == 2 and p["order"] == 2
    assert p["tau"] == 0.01 and p["end_time"] == 0.095 and p["xr"] == 15.75 and p["save_rate"] == 2
    assert p["nic"] == 1 and p["ic"][0] == 3  # GPE_IC_RING
    assert p["ring_r0"] == 4.0 and p["ring_plane"] == "xy"


def test_ic_products_and_single_precision(ring_dir):
    (ring_dir / "ic.in").write_text("  init_cond = fermi() * vortex_line(vl1)\n")
    pin = (ring_dir / "parameters.in").read_text()
    pin = pin.replace("  !integer, parameter :: pr = selected_real_kind(6,37)\n  integer, parameter :: pr = "
                      "selected_real_kind(15,307)", "  integer, parameter :: pr = selected_real_kind(6,37)")
    (ring_dir / "parameters.in").write_text(pin)
    p = json.loads(run_host(ring_dir, "--parse-only").stdout)
    assert p["pr"] == 4 and p["nic"] == 2 and p["ic"][:2] == [1, 2] and p["line_dir"] == "z"


def test_pade_pulse_and_closed_form_factors(ring_dir):
    # pade_pulse_ring, vortex_pair, sphere, sphere2 and wall (src/ic.f90:518-709)
    (ring_dir / "ic.in").write_text("! Pade rarefaction pulse\n"
                                    "  init_cond = pade_pulse_ring('pulse', 0.5_pr, -1.0_pr, 2.0_pr, 0.0_pr) * "
                                    "vortex_pair() * wall()\n")
    p = json.loads(run_host(ring_dir, "--parse-only").stdout)
    assert p["nic"] == 3 and p["ic"][:3] == [6, 8, 11] and p["pulse"] == [0.5, -1.0, 2.0, 0.0]
    (ring_dir / "ic.in").write_text("  init_cond = pade_pulse_ring('ring', 0.0, 0.0, 0.0, 6.5) * sphere2() * sphere()\n")
    p = json.loads(run_host(ring_dir, "--parse-only").stdout)
    assert p["nic"] == 3 and p["ic"][:3] == [7, 10, 9] and p["pulse"] == [0.0, 0.0, 0.0, 6.5]


@pytest.mark.parametrize("expr, msg", [
    ("pade_pulse_ring('wave', 0.0, 0.0, 0.0, 1.0)", "pulse_or_ring must be 'pulse' or 'ring'"),
    ("pade_pulse_ring('pulse', 0.0, 0.0, 1.0)", "pade_pulse_ring takes (pulse_or_ring, x0, y0, z0, r0)"),
    ("pade_pulse_ring('pulse', 0, 0, 0, 1) * pade_pulse_ring('ring', 0, 0, 0, 2)", "different arguments"),
    ("vortex_sheet()", "is not supported"),
])
def test_bad_ic_products_are_emergency_stops(ring_dir, expr, msg):
    (ring_dir / "ic.in").write_text(f"  init_cond = {expr}\n")
    r = run_host(ring_dir, "--parse-only")
    assert r.returncode != 0
    assert msg in (ring_dir / "ERROR").read_text()


@pytest.mark.parametrize("group, flag", [("io_params", "save_contour"), ("io_params", "save_average"),
                                         ("io_params", "save_pdf"), ("io_params", "save_vcf"),
                                         ("io_params", "save_ll"), ("io_params", "save_zeros"),
                                         ("misc_params", "diagnostic"), ("misc_params", "pp_filtered_surface")])
def test_unbuilt_diagnostics_are_emergency_stops(ring_dir, group, flag):
    # a run that asks for a diagnostic this host does not write stops with
    # ERROR (src/error.f90:24-46) instead of silently writing fewer files
    t = (ring_dir / "run.in").read_text()
    t = t.replace(f"  {flag}  = .false.\n", "")
    head = t.index(f"&{group}") + len(f"&{group}") + 1
    (ring_dir / "run.in").write_text(t[:head] + f"  {flag} = .true.\n" + t[head:])
    r = run_host(ring_dir, "--parse-only")
    assert r.returncode != 0
    assert f"{flag} = .true. needs" in (ring_dir / "ERROR").read_text()


def test_unknown_scheme_is_an_emergency_stop(ring_dir):
    t = (ring_dir / "run.in").read_text().replace("'rk4'", "'rk9'")
    (ring_dir / "run.in").write_text(t)
    r = run_host(ring_dir, "--parse-only")
    assert r.returncode != 0
    assert "Unrecognised time stepping scheme" in (ring_dir / "ERROR").read_text()


def test_missing_namelist_is_an_emergency_stop(ring_dir):
    t = (ring_dir / "run.in").read_text()
    (ring_dir / "run.in").write_text(t[: t.index("&misc_params")])
    r = run_host(ring_dir, "--parse-only")
    assert r.returncode != 0
    assert "error reading namelist misc_params" in (ring_dir / "ERROR").read_text()


def test_imprint_without_a_vortex_line_is_an_emergency_stop(ring_dir):
    t = (ring_dir / "run.in").read_text().replace("imprint_vl          = .false.", "imprint_vl          = .true.")
    (ring_dir / "run.in").write_text(t)
    pin = (ring_dir / "parameters.in").read_text()
    start = pin.index("  type (line_param)")
    end = pin.index("  type (ring_param)")
    (ring_dir / "parameters.in").write_text(pin[:start] + pin[end:])
    r = run_host(ring_dir)
    assert r.returncode != 0
    assert "imprint_vl=.true. but parameters.in has no vl1" in (ring_dir / "ERROR").read_text()
