"""Device FFT diagnostics (gpe_condensed / gpe_filtered) against the numpy
restatement of condensed_particles, spectrum and filtered_surface
(oracle/fft_diag.py, src/io.f90:304-714)."""
from __future__ import annotations

import numpy as np
import pytest

from gpe_b200 import ic
from gpe_b200.solver import RunParams, Solver
from oracle import fft_diag as D

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _states():
    rp1 = RunParams(nx=32, ny=28, nz=24, xr=7.75, yr=6.75, zr=5.75, bcs=1, order=4)
    rp2 = RunParams(nx=48, ny=40, nz=36, xr=11.75, yr=9.75, zr=8.75, bcs=2, order=2)
    rp3 = RunParams(nx=40, ny=40, nz=40, xr=9.75, yr=9.75, zr=9.75, bcs=1, order=4)
    return [
        ("random_phase", rp1, ic.random_phase(rp1, seed=9, kc=1.2)),
        ("ring", rp2, ic.vortex_ring(rp2, "xy", r0=3.0)),
        ("ring_x_random", rp3, ic.vortex_ring(rp3, "xz", r0=2.5) * ic.random_phase(rp3, seed=4, kc=2.0)),
    ]


@pytest.mark.parametrize("case", [0, 1, 2])
@pytest.mark.parametrize("storage", ["c128", "c64"])
def test_condensed_and_spectrum_match_oracle(gpu, case, storage):
    name, rp, psi = _states()[case]
    rp = rp.replace(storage=storage)
    s = Solver(rp)
    s.set_state(psi)
    # the oracle sees exactly the stored state (complex64 rounding included)
    stored = s.get_state().astype(np.complex128)
    dev = s.condensed(spectrum=True)
    rec, a = D.condensed_particles(stored, rp.xr, rp.yr, rp.zr)
    for k in ("M", "tot", "temp", "temp2", "H", "mass_density"):
        assert dev[k] == pytest.approx(rec[k], rel=TOL), k
    # n0 is a single spectral coefficient: compare against the total mass scale
    scale = np.sum(np.abs(stored) ** 2)
    assert abs(dev["n0"] - rec["n0"]) <= TOL * scale
    eta, nharm, F = D.spectrum(a)
    assert np.array_equal(dev["nharm"], nharm)
    np.testing.assert_allclose(dev["eta"], eta, rtol=TOL, atol=TOL * scale / stored.size)
    np.testing.assert_allclose(dev["F"], F, rtol=TOL, atol=TOL * scale)
    s.close()


def test_condensed_is_deterministic(gpu):
    _, rp, psi = _states()[0]
    s = Solver(rp)
    s.set_state(psi)
    r1 = s.condensed(spectrum=True)
    r2 = s.condensed(spectrum=True)
    for k, v in r1.items():
        assert np.array_equal(np.asarray(v), np.asarray(r2[k])), k
    s.close()


@pytest.mark.parametrize("case", [0, 1])
@pytest.mark.parametrize("m,kc", [(1.0, 4.0), (0.5, 9.0)])
def test_filtered_matches_oracle(gpu, case, m, kc):
    _, rp, psi = _states()[case]
    s = Solver(rp)
    s.set_state(psi)
    out = s.filtered(kc, m=m)
    _, a = D.condensed_particles(psi, rp.xr, rp.yr, rp.zr)
    ref = D.filtered_surface(a, m, kc)
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err <= TOL
    out32 = s.filtered(kc, m=m, dtype=np.complex64)
    assert np.array_equal(out32, out.astype(np.complex64))
    s.close()


def test_condensed_argument_checks(gpu):
    _, rp, psi = _states()[0]
    s = Solver(rp)
    s.set_state(psi)
    from gpe_b200 import _lib as L
    import ctypes as C

    info = L.GpeCondensedInfo()
    F = np.zeros(3)
    assert s.lib.gpe_condensed(s.h, C.byref(info), None, None, F.ctypes.data, 3) == L.GPE_ERR_BADARG
    out = np.zeros(psi.shape, dtype=np.complex128)
    assert s.lib.gpe_filtered(s.h, 1.0, 0.0, out.ctypes.data, L.GPE_C128) == L.GPE_ERR_BADARG
    s.close()
