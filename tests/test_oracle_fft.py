"""Pin the FFT-diagnostics oracle (oracle/fft_diag.py) with analytic cases:
transforms of constants and single Fourier modes, Parseval, shell counts
and the filter's action on single modes (src/io.f90:304-714)."""
import numpy as np
import pytest

from oracle import fft_diag as D


def _mode(shape, m):
    nz, ny, nx = shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ph = 2 * np.pi * (m[0] * i / nx + m[1] * j / ny + m[2] * k / nz)
    return np.exp(1j * ph)


def test_fft_normalisation_and_sign():
    shape = (6, 5, 8)
    psi = _mode(shape, (1, 0, 0))
    a = D.fft(psi, "forward")
    n = psi.size
    # exp(+2 pi i x/nx) lands on index +1 with the exp(-i k x) forward sign
    assert abs(a[0, 0, 1] - np.sqrt(n)) < 1e-12
    a[0, 0, 1] = 0
    assert np.max(np.abs(a)) < 1e-12
    back = D.fft(D.fft(psi, "forward"), "backward")
    assert np.max(np.abs(back - psi)) < 1e-13


def test_uniform_state():
    shape = (8, 6, 10)
    psi = np.ones(shape, dtype=np.complex128)
    rec, a = D.condensed_particles(psi, 2.0, 1.5, 3.0)
    n = psi.size
    assert rec["n0"] == pytest.approx(n, rel=1e-14)
    dx, dy, dz = D.spacing(10, 2.0), D.spacing(6, 1.5), D.spacing(8, 3.0)
    assert rec["M"] == pytest.approx(n * dx * dy * dz, rel=1e-14)
    assert rec["rho0"] == pytest.approx(1.0, rel=1e-14)
    eta, nharm, F = D.spectrum(a)
    assert np.all(np.abs(eta) < 1e-20) and np.all(np.abs(F) < 1e-20)


def test_parseval_and_mass():
    rng = np.random.default_rng(3)
    psi = rng.normal(size=(7, 9, 12)) + 1j * rng.normal(size=(7, 9, 12))
    a = D.fft(psi, "forward")
    assert np.sum(np.abs(a) ** 2) == pytest.approx(np.sum(np.abs(psi) ** 2), rel=1e-13)


def test_single_mode_spectrum():
    shape = (16, 16, 16)
    m = (3, 4, 0)  # |k| = 5 in index units
    psi = _mode(shape, m)
    rec, a = D.condensed_particles(psi, 7.5, 7.5, 7.5)
    n = psi.size
    assert rec["n0"] < 1e-20
    eta, nharm, F = D.spectrum(a)
    # F(kk) = N for kk >= 5, 0 below
    assert np.all(np.abs(F[:4]) < 1e-12)
    assert np.allclose(F[4:], n, rtol=1e-13)
    # |log2(5 / (2 pi))| = 0.33 -> shell 1 holds the mode
    assert eta[0] * nharm[0] == pytest.approx(n, rel=1e-13)
    assert np.all(np.abs(eta[1:]) < 1e-20)


def test_shell_counts_partition_the_grid():
    shape = (12, 10, 14)
    k2 = (D.k2_index(14)[None, None, :] + D.k2_index(10)[None, :, None] + D.k2_index(12)[:, None, None])
    a = np.ones(shape, dtype=np.complex128)
    _, nharm, _ = D.spectrum(a)
    r = np.sqrt(k2[k2 > 0].astype(float)) / (2 * np.pi)
    expect = np.bincount(np.floor(np.abs(np.log2(r))).astype(int), minlength=7)[:7]
    assert np.array_equal(nharm, expect)


def test_filter_on_single_modes():
    shape = (16, 16, 16)
    kc = 6.0
    for m in [(2, 0, 0), (3, 4, 0), (6, 0, 0), (7, 1, 0)]:
        psi = _mode(shape, m)
        _, a = D.condensed_particles(psi, 7.5, 7.5, 7.5)
        out = D.filtered_surface(a, 1.0, kc)
        k2 = sum(c * c for c in m)
        f = max(1.0 - k2 / kc ** 2, 0.0)
        assert np.max(np.abs(out - f * psi)) < 1e-12
