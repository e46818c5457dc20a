"""CPU restatement of the reference's FFT diagnostics -- TEST INFRASTRUCTURE
ONLY (the oracle for gpe_condensed / gpe_filtered).  Nothing in the product
path imports this module.

Restates, in numpy, for a single process:
  * fft                  src/ic.f90:910-939   (DFT normalised by 1/sqrt(N) both ways)
  * condensed_particles  src/io.f90:304-395   (n0, mass, tot, temp, temp2, H)
  * mass                 src/variables.f90:608-628
  * spectrum             src/io.f90:668-714   (eta, nharm, F)
  * filtered_surface     src/io.f90:524-571   (low-pass + inverse transform)

numpy's fftn has the FFTW sign convention of 2DECOMP&FFT's forward
transform (exp(-i k x)); its sums run in a different order from the
reference's loops, so agreement is to rounding.  Parity of these routines is
unpinned by reference outputs (the reference ships none and cannot be built
here); tests/test_oracle_fft.py pins the restatement with analytic cases.
"""
from __future__ import annotations

import numpy as np

PI = 3.1415926535897932384626433832795
NSHELLS = 7


def fft(var: np.ndarray, direction: str) -> np.ndarray:
    """src/ic.f90:910-939: forward = exp(-i k x) sum, backward = exp(+i k x)
    sum, both divided by sqrt(nx ny nz)."""
    n = var.size
    if direction == "forward":
        out = np.fft.fftn(var)
    elif direction == "backward":
        out = np.fft.ifftn(var) * n
    else:
        raise ValueError("ERROR: Not a valid direction for FFT!")
    return out / np.sqrt(float(n))


def k2_index(n: int) -> np.ndarray:
    """Squared spectral index distance on one axis (src/io.f90:547-565)."""
    n1 = n - 1
    i = np.arange(n, dtype=np.int64)
    return np.where(i <= n1 // 2 + 1, i * i, (n1 - i + 1) ** 2)


def kq_axis(n: int, nx: int, d: float) -> np.ndarray:
    """The per-axis Laplacian symbol on the reference's k grid, kx = -pi + i dk
    with dk = 2 pi/(nx - 1) on every axis (src/io.f90:323-324, 345-357)."""
    kc = PI
    dk = 2.0 * kc / float(nx - 1)
    k = -kc + np.arange(n, dtype=np.float64) * dk
    return ((-2.0 * np.cos(2.0 * k * d) + 32.0 * np.cos(k * d)) - 30.0) / (d * d)


def spacing(n: int, r: float) -> float:
    """get_grid's dx = 2 r / (n - 1) (src/ic.f90:43-51)."""
    return (r - (-r)) / (n - 1)


def mass(psi: np.ndarray, dx: float, dy: float, dz: float) -> float:
    """src/variables.f90:608-628."""
    return ((float(np.sum(np.abs(psi) ** 2)) * dx) * dy) * dz


def condensed_particles(psi: np.ndarray, xr: float, yr: float, zr: float):
    """src/io.f90:304-381: returns (record dict, a = fft(psi, 'forward'))."""
    nz, ny, nx = psi.shape
    V = nx * ny * nz
    dx, dy, dz = spacing(nx, xr), spacing(ny, yr), spacing(nz, zr)
    a = fft(psi.astype(np.complex128), "forward")
    n0 = float(np.abs(a[0, 0, 0]) ** 2)
    M = mass(psi.astype(np.complex128), dx, dy, dz)
    rho0 = n0 / V
    kx, ky, kz = kq_axis(nx, nx, dx), kq_axis(ny, nx, dy), kq_axis(nz, nx, dz)
    k2 = -(1.0 / 12.0) * ((kx[None, None, :] + ky[None, :, None]) + kz[:, None, None])
    keep = k2 != 0.0
    k2 = k2[keep]
    tot = float(np.sum((k2 + rho0) / (k2 * k2 + 2.0 * rho0 * k2)))
    temp = (M - n0) / tot
    E0 = (1.0 / float(2 * V)) * (M ** 2 + (M - n0) ** 2)
    H = E0 + temp * float(V - 1)
    vol8 = ((8.0 * xr) * yr) * zr
    temp2 = ((M / vol8) - (n0 / V)) / tot
    rec = dict(M=M, n0=n0, rho0=rho0, tot=tot, temp=temp, temp2=temp2, H=H, mass_density=M / vol8)
    return rec, a


def spectrum(a: np.ndarray):
    """src/io.f90:668-714: (eta per shell divided by its count, nharm, F[kk-1])."""
    nz, ny, nx = a.shape
    k2 = k2_index(nx)[None, None, :] + k2_index(ny)[None, :, None] + k2_index(nz)[:, None, None]
    v = np.abs(a) ** 2
    rk = np.sqrt(k2.astype(np.float64))
    nonzero = rk != 0.0
    F = np.array([np.sum(v[nonzero & (rk <= float(kk))]) for kk in range(1, nx // 2 + 1)])
    with np.errstate(divide="ignore"):
        log2k = np.log(0.5 * rk / PI) / np.log(2.0)
    al = np.abs(log2k)
    eta = np.zeros(NSHELLS)
    nharm = np.zeros(NSHELLS, dtype=np.int64)
    for m in range(1, NSHELLS + 1):
        sel = nonzero & (al < float(m)) & (al >= float(m - 1))
        eta[m - 1] = np.sum(v[sel])
        nharm[m - 1] = int(np.count_nonzero(sel))
    for m in range(NSHELLS):
        if eta[m] != 0.0:
            eta[m] = eta[m] / float(nharm[m])
    return eta, nharm, F


def filtered_surface(a: np.ndarray, m: float, filter_kc: float) -> np.ndarray:
    """src/io.f90:545-571: a * max(1 - m k2/kc^2, 0), transformed back."""
    nz, ny, nx = a.shape
    k2 = k2_index(nx)[None, None, :] + k2_index(ny)[None, :, None] + k2_index(nz)[:, None, None]
    f = np.maximum(1.0 - (m * k2.astype(np.float64) / filter_kc ** 2), 0.0)
    return fft(a * f, "backward")
