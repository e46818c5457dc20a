"""Initial conditions on the host (numpy), restating the reference's ic.f90
for the products a run.in/ic.in pair can ask for, plus the seeded
random-phase state used by the 256^3 benchmark workload.

Arrays have shape (nz, ny, nx) (the reference's psi(0:nx1,0:ny1,0:nz1)
memory order).  The grid is the reference's node-inclusive grid
x_i = -xr + i*2xr/(nx-1) (src/ic.f90:32-69).
"""
from __future__ import annotations

import numpy as np

PI = 3.1415926535897932384626433832795


def grid(n: int, r: float):
    """get_grid (src/ic.f90:43-66) for one axis: (coordinates, spacing)."""
    lo = -r
    d = (r - lo) / (n - 1)
    return lo + np.arange(n, dtype=np.float64) * d, d


def _mesh(p):
    x, _ = grid(p.nx, p.xr)
    y, _ = grid(p.ny, p.yr)
    z, _ = grid(p.nz, p.zr)
    return x[None, None, :], y[None, :, None], z[:, None, None]


def get_rr(r):
    """get_rr (src/ic.f90:893-906): R(r)/r of the Pade vortex core."""
    r2 = r * r
    r4 = r2 * r2
    return np.sqrt((0.3437 + 0.0286 * r2) / ((1.0 + 0.3333 * r2) + 0.0286 * r4))


def vortex_ring(p, plane="xy", x0=0.0, y0=0.0, z0=0.0, r0=4.0, amp=0.0, mm=0, r1=0.0, kk=0, dir=1.0):
    """vortex_ring (src/ic.f90:357-514): two Pade-core branches with opposite
    winding a distance r0 from the ring axis."""
    X, Y, Z = _mesh(p)
    if plane == "xy":
        u, v, w, u0, v0, w0 = X, Y, Z, x0, y0, z0
    elif plane == "xz":
        u, v, w, u0, v0, w0 = X, Z, Y, x0, z0, y0
    elif plane == "yz":
        u, v, w, u0, v0, w0 = Y, Z, X, y0, z0, x0
    else:
        raise ValueError("ERROR: Unrecognised vortex ring plane.")
    sc = p.scal
    theta = np.arctan2(v - v0, u - u0)
    s = np.sqrt((u - u0) ** 2 + (v - v0) ** 2) - r1 * np.sin(float(kk) * theta)
    dist = amp * np.cos(float(mm) * theta)
    pp = w - r1 * np.cos(float(kk) * theta)
    A = sc * (pp - w0)
    Bp = sc * ((s + r0) - dist)
    Bm = sc * ((s - r0) - dist)
    d1 = np.sqrt(A * A + Bp * Bp)
    d2 = np.sqrt(A * A + Bm * Bm)
    z1 = (A + 0.0 * Bp) + 1j * (dir * Bp)
    z2 = (A - 0.0 * Bm) - 1j * (dir * Bm)
    out = ((get_rr(d1) * z1) * get_rr(d2)) * z2
    return np.ascontiguousarray(np.broadcast_to(out, (p.nz, p.ny, p.nx)), dtype=np.complex128)


def _line_geom(p, x0, y0, z0, amp1, amp2, ll, sgn, dir):
    """get_r (src/ic.f90:735-800) and get_theta (src/ic.f90:824-889)."""
    X, Y, Z = _mesh(p)
    eps = np.finfo(np.float64).eps
    safe1 = safe2 = 0.0
    if abs(ll) < eps:
        if abs(amp1) >= eps or abs(amp2) >= eps:
            raise ValueError("ERROR: vortex line disturbance wavelength is zero, but amplitude is non-zero.")
        safe1 = safe2 = 1.0
    if dir == "x":
        a = Y - y0 - amp1 * np.sin(2.0 * PI * (X - x0) / (ll + safe1))
        b = Z - z0 - amp2 * np.cos(2.0 * PI * (X - x0) / (ll + safe2))
    elif dir == "y":
        a = Z - z0 - amp1 * np.sin(2.0 * PI * (Y - y0) / (ll + safe1))
        b = X - x0 - amp2 * np.cos(2.0 * PI * (Y - y0) / (ll + safe2))
    elif dir == "z":
        a = X - x0 - amp1 * np.sin(2.0 * PI * (Z - z0) / (ll + safe1))
        b = Y - y0 - amp2 * np.cos(2.0 * PI * (Z - z0) / (ll + safe2))
    else:
        raise ValueError("vortex line direction must be x, y or z")
    sc = p.scal
    r = np.sqrt(sc * (a * a) + sc * (b * b))
    theta = sgn * np.arctan2(sc * b, sc * a)
    return np.broadcast_to(r, (p.nz, p.ny, p.nx)), np.broadcast_to(theta, (p.nz, p.ny, p.nx))


def vortex_line(p, x0=0.0, y0=0.0, z0=0.0, amp1=0.0, amp2=0.0, ll=0.0, sgn=1.0, dir="z",
                imprint_phase=False):
    """vortex_line (src/ic.f90:332-353) with core 1 - exp(-0.7 r^1.15)
    (src/ic.f90:314-328)."""
    r, th = _line_geom(p, x0, y0, z0, amp1, amp2, ll, sgn, dir)
    a = 1.0 if imprint_phase else 1.0 - np.exp(-0.7 * r ** 1.15)
    return np.ascontiguousarray(a * np.cos(th) + 1j * (a * np.sin(th)), dtype=np.complex128)


def vortex_line_pade(p, x0=0.0, y0=0.0, z0=0.0, amp1=0.0, amp2=0.0, ll=0.0, sgn=1.0, dir="z"):
    """Vortex line with the Pade core R(r) = r*get_rr(r) of the ring
    (src/ic.f90:893-906) instead of the exponential core."""
    r, th = _line_geom(p, x0, y0, z0, amp1, amp2, ll, sgn, dir)
    a = r * get_rr(r)
    return np.ascontiguousarray(a * np.cos(th) + 1j * (a * np.sin(th)), dtype=np.complex128)


def vtrap(p):
    """Vtrap (src/ic.f90:713-731)."""
    X, Y, Z = _mesh(p)
    v = 0.5 * (((p.omx * p.omx) * (X * X) + (p.omy * p.omy) * (Y * Y)) + (p.omz * p.omz) * (Z * Z))
    return np.ascontiguousarray(np.broadcast_to(v, (p.nz, p.ny, p.nx)))


def fermi(p):
    """fermi (src/ic.f90:278-310): Thomas-Fermi sqrt(max(mu - V, 0)/g)."""
    f = (p.mu - vtrap(p)) / p.g
    out = np.where(f >= 0.0, np.sqrt(np.maximum(f, 0.0)), 0.0)
    return out.astype(np.complex128)


# get_consts (src/ic.f90:563-585): the published Pade coefficients a(1..9),
# velocity U and momentum m of the vortex ring and the rarefaction pulse
_PADE = {
    "ring": ((-1.1, 0.0170524, 0.0289452, -0.953, -0.0049767, -0.0594346, 0.04, 0.21, 0.00612), 0.6, 8.97),
    "pulse": ((-0.79792, 0.00388059, 0.00882276, -0.7981, -0.012783, -0.0574092, 0.0399, 0.199, 0.0058), 0.63,
              8.37),
}


def pade_pulse_ring(p, pulse_or_ring="pulse", x0=0.0, y0=0.0, z0=0.0, r0=0.0):
    """pade_pulse_ring (src/ic.f90:518-587): the Pade approximation of a
    rarefaction pulse ('pulse') or an axisymmetric vortex ring ('ring')
    moving along x, centred at x0 with its axis through (y0, z0), radius r0
    (N. G. Berloff, J. Phys. A 37, 1617 (2004))."""
    a, U, m = _PADE[pulse_or_ring]
    X, Y, Z = _mesh(p)
    pw = 7.0 / 4.0
    one_2u = 1.0 - 2.0 * (U * U)
    ma9 = m * a[8] ** pw
    s = np.sqrt((Y - y0) * (Y - y0) + (Z - z0) * (Z - z0))  # get_s (src/ic.f90:804-820)
    xs = X - x0
    x2 = xs * xs
    s2 = (s - r0) * (s - r0)
    t = x2 + one_2u * s2
    denom = (((1.0 + a[7] * x2) + a[6] * s2) + a[8] * (t * t)) ** pw
    uu = 1.0 + ((((a[0] + a[2] * x2) + a[1] * s2) + (ma9 * U) * (2.0 * x2 - one_2u * s2)) * t) / denom
    vv = (xs * (((a[3] + a[5] * x2) + a[4] * s2) - ma9 * (t * t))) / denom
    return np.ascontiguousarray(np.broadcast_to(uu + 1j * vv, (p.nz, p.ny, p.nx)), dtype=np.complex128)


def vortex_pair(p):
    """vortex_pair (src/ic.f90:591-636): Pade approximation of a vortex pair
    in the x-y plane, the same in every z plane."""
    a0, a1, a2 = -1.14026, -0.150112, -0.0294564
    b0, b1, b2 = -0.830953, -0.108296, -0.073641
    c0, c1, c2, c3, c4 = 0.35022, 0.03032, 0.15905, 0.04123, 0.01402
    X, Y, _ = _mesh(p)
    x2, y2 = X * X, Y * Y
    denom = ((((1.0 + c0 * x2) + c1 * (x2 * x2)) + c2 * y2) + (c3 * x2) * y2) + c4 * (y2 * y2)
    v = (1.0 + ((a0 + a1 * x2) + a2 * y2) / denom) + 1j * ((X * ((b0 + b1 * x2) + b2 * y2)) / denom)
    return np.ascontiguousarray(np.broadcast_to(v, (p.nz, p.ny, p.nx)), dtype=np.complex128)


def sphere(p):
    """sphere (src/ic.f90:640-662): 0.5 (1 + tanh(r - rad - eps1)), rad = 10, eps1 = 2."""
    X, Y, Z = _mesh(p)
    v = 0.5 * (1.0 + np.tanh((np.sqrt((X * X + Y * Y) + Z * Z) - 10.0) - 2.0))
    return np.ascontiguousarray(np.broadcast_to(v, (p.nz, p.ny, p.nx)), dtype=np.complex128)


def sphere2(p):
    """sphere2 (src/ic.f90:666-684): amp exp(-r^2/width), amp = 100, width = 10."""
    X, Y, Z = _mesh(p)
    v = 100.0 * np.exp(-((X * X + Y * Y) + Z * Z) / 10.0)
    return np.ascontiguousarray(np.broadcast_to(v, (p.nz, p.ny, p.nx)), dtype=np.complex128)


def wall(p):
    """wall (src/ic.f90:688-709): 0 for z <= pos, else 1, pos = -30."""
    _, _, Z = _mesh(p)
    v = np.where(Z <= -30.0, 0.0, 1.0)
    return np.ascontiguousarray(np.broadcast_to(v, (p.nz, p.ny, p.nx)), dtype=np.complex128)


_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, idx: np.ndarray) -> np.ndarray:
    """SplitMix64 (S. Vigna) output for counter values idx under seed."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + (idx.astype(np.uint64) + np.uint64(1)) * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def random_phase(p, seed: int = 1234, kc: float = 1.5):
    """Seeded random-phase state: psi_hat(k) = sqrt(n(k)) e^{i theta_k},
    n(k) = const for |k| < kc, theta_k uniform on [0, 2 pi) from SplitMix64
    over the linear mode index; inverse FFT; rescaled to mean density 1.
    k = 2 pi m / L with L = n dx the periodic length of each axis.  (This is
    the benchmark's stated spectrum, not the reference's random_phase(),
    whose phases come from an unseeded gfortran RNG, src/ic.f90:213-224.)"""
    _, dx = grid(p.nx, p.xr)
    _, dy = grid(p.ny, p.yr)
    _, dz = grid(p.nz, p.zr)
    kx = 2.0 * PI * np.fft.fftfreq(p.nx, d=dx)
    ky = 2.0 * PI * np.fft.fftfreq(p.ny, d=dy)
    kz = 2.0 * PI * np.fft.fftfreq(p.nz, d=dz)
    k2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    mask = k2 < kc * kc
    idx = np.arange(p.nx * p.ny * p.nz, dtype=np.uint64).reshape(p.nz, p.ny, p.nx)
    u = (splitmix64(seed, idx) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    spec = np.where(mask, np.exp(1j * (2.0 * PI * u)), 0.0)
    psi = np.fft.ifftn(spec)
    psi *= 1.0 / np.sqrt(np.mean(np.abs(psi) ** 2))
    return np.ascontiguousarray(psi, dtype=np.complex128)


# ---------------------------------------------------------------------------
# Device-side initial conditions: specs for gpe_set_ic / gpe_pool_submit_ic


def device_spec(*factors, ring=None, line=None, pulse=None, seed: int = 1234, kc: float = 1.5):
    """Build a gpe_ic spec: the product of the named factors ("uniform",
    "fermi", "line", "ring", "line_pade", "random_phase", "pade_pulse",
    "pade_ring", "vortex_pair", "sphere", "sphere2", "wall").  ring / line
    are dicts with the fields of ring_param / line_param
    (src/parameters.in); pulse = dict(x0, y0, z0, r0), the arguments of
    pade_pulse_ring."""
    from . import _lib as L

    codes = {"uniform": L.GPE_IC_UNIFORM, "fermi": L.GPE_IC_FERMI, "line": L.GPE_IC_LINE,
             "ring": L.GPE_IC_RING, "line_pade": L.GPE_IC_LINE_PADE, "random_phase": L.GPE_IC_RANDOM_PHASE,
             "pade_pulse": L.GPE_IC_PADE_PULSE, "pade_ring": L.GPE_IC_PADE_RING,
             "vortex_pair": L.GPE_IC_VORTEX_PAIR, "sphere": L.GPE_IC_SPHERE, "sphere2": L.GPE_IC_SPHERE2,
             "wall": L.GPE_IC_WALL}
    spec = L.GpeIC()
    spec.nfactors = len(factors)
    for q, f in enumerate(factors):
        spec.factor[q] = codes[f]
    r = dict(plane="xy", x0=0.0, y0=0.0, z0=0.0, r0=4.0, amp=0.0, mm=0, r1=0.0, kk=0, dir=1.0)
    r.update(ring or {})
    for k, v in r.items():
        setattr(spec.ring, k, v.encode() if k == "plane" else v)
    ln = dict(x0=0.0, y0=0.0, z0=0.0, amp1=0.0, amp2=0.0, ll=0.0, sgn=1.0, dir="z", imprint_phase=0)
    ln.update(line or {})
    for k, v in ln.items():
        setattr(spec.line, k, v.encode() if k == "dir" else (int(v) if k == "imprint_phase" else v))
    pu = dict(x0=0.0, y0=0.0, z0=0.0, r0=0.0)
    pu.update(pulse or {})
    for k, v in pu.items():
        setattr(spec.pulse, k, float(v))
    spec.seed = int(seed)
    spec.kc = float(kc)
    return spec
