"""Pin the CPU oracle against analytic known answers derived from the
reference's formulas (the reference ships no tests or golden vectors):

  * the FD operators of src/derivs.f90 are exact on low-degree polynomials
    and have the closed-form plane-wave symbols (the reference uses the
    4th-order symbol itself at src/io.f90:355-361);
  * reflective BCs (src/derivs.f90:365-394) equal periodic BCs on the even
    extension of the field;
  * the schemes of src/solve.f90 multiply a Fourier mode of the linear
    equation by their exact amplification polynomials (tests/golden/
    kat_polys.json, derived with exact rationals from the tableaux);
  * rkqs step control (src/solve.f90:173-229) follows Numerical Recipes
    16.2 on a scripted error sequence;
  * uniform states are stationary; the quadrature of src/variables.f90:
    730-840 is exact on cubics; energy of a plane wave has a closed form.
"""
from __future__ import annotations

import json
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

from gpe_b200 import ic
from gpe_b200.solver import RunParams
from oracle.pyoracle import Oracle

GOLD = Path(__file__).resolve().parent / "golden"
POLYS = {k: v for k, v in json.loads((GOLD / "kat_polys.json").read_text()).items()}


def poly(name, z):
    return sum(float(Fraction(c)) * z ** k for k, c in enumerate(POLYS[name]))


def rp_small(**kw):
    base = dict(nx=16, ny=12, nz=10, xr=4.0, yr=3.0, zr=2.5, tau=0.01, scheme="rk4", eqn_to_solve=4,
                bcs=1, order=4, g=0.0, mu=0.0)
    base.update(kw)
    return RunParams(**base)


def mesh(o):
    x, y, z, d = o.grid()
    return x[None, None, :], y[None, :, None], z[:, None, None], d


def symbol(order, k, h):
    if order == 2:
        return (2 * np.cos(k * h) - 2) / h ** 2
    return (-2 * np.cos(2 * k * h) + 32 * np.cos(k * h) - 30) / (12 * h ** 2)


@pytest.mark.parametrize("order", [2, 4])
def test_plane_wave_symbol(order):
    o = Oracle(rp_small(order=order))
    X, Y, Z, d = mesh(o)
    rp = o.rp
    k = [2 * np.pi * m / (n * h) for m, n, h in ((3, rp.nx, d[0]), (2, rp.ny, d[1]), (1, rp.nz, d[2]))]
    psi = np.exp(1j * (k[0] * X + k[1] * Y + k[2] * Z)) * np.ones(o.shape)
    lam = sum(symbol(order, kk, h) for kk, h in zip(k, d))
    np.testing.assert_allclose(o.laplacian(psi), lam * psi, rtol=0, atol=1e-12)
    # first derivative symbol (derivs.f90:43, 54-57)
    kx, h = k[0], d[0]
    s1 = 1j * np.sin(kx * h) / h if order == 2 else 1j * (8 * np.sin(kx * h) - np.sin(2 * kx * h)) / (6 * h)
    np.testing.assert_allclose(o.deriv_x(psi), s1 * psi, rtol=0, atol=1e-12)


@pytest.mark.parametrize("order,deg", [(2, 3), (4, 5)])
def test_polynomial_exactness_interior(order, deg):
    o = Oracle(rp_small(order=order, bcs=2))
    X, Y, Z, d = mesh(o)
    f = (X ** deg + 0.5 * Y ** (deg - 1) - 0.25 * Z ** deg) * np.ones(o.shape)
    exact = (deg * (deg - 1) * X ** (deg - 2) + 0.5 * (deg - 1) * (deg - 2) * Y ** (deg - 3)
             - 0.25 * deg * (deg - 1) * Z ** (deg - 2)) * np.ones(o.shape)
    lap = o.laplacian(f.astype(np.complex128)).real
    r = order // 2
    sl = (slice(r, -r), slice(r, -r), slice(r, -r))
    np.testing.assert_allclose(lap[sl], exact[sl], rtol=1e-10, atol=1e-9)


@pytest.mark.parametrize("order", [2, 4])
def test_reflective_equals_even_extension(order):
    rng = np.random.default_rng(7)
    rp = rp_small(order=order, bcs=2, nx=9, ny=8, nz=7)
    o = Oracle(rp)
    f = rng.standard_normal(o.shape) + 1j * rng.standard_normal(o.shape)
    lap_r = o.laplacian(f)
    # even extension about the end nodes -> period 2(n-1) in every axis
    g = f
    for ax in range(3):
        n = g.shape[ax]
        idx = np.r_[np.arange(n), np.arange(n - 2, 0, -1)]
        g = np.take(g, idx, axis=ax)
    _, _, _, d = o.grid()
    nz2, ny2, nx2 = g.shape
    rpp = rp_small(order=order, bcs=1, nx=nx2, ny=ny2, nz=nz2,
                   xr=d[0] * (nx2 - 1) / 2, yr=d[1] * (ny2 - 1) / 2, zr=d[2] * (nz2 - 1) / 2)
    op = Oracle(rpp)
    lap_p = op.laplacian(g)[: rp.nz, : rp.ny, : rp.nx]
    np.testing.assert_allclose(lap_r, lap_p, rtol=0, atol=1e-10)


@pytest.mark.parametrize("eqn", [1, 2, 4])
def test_uniform_state_is_stationary(eqn):
    # eqn 1: (1-|psi|^2) psi = 0 at |psi| = 1; eqn 4 with V = 0, g = mu = 1;
    # eqn 2 rotates the phase at rate -1: check against exp(-i t) instead.
    rp = rp_small(eqn_to_solve=eqn, g=1.0, mu=1.0, bcs=2, order=4)
    o = Oracle(rp)
    psi = np.ones(o.shape, np.complex128)
    rhs = o.get_rhs(psi)
    if eqn == 2:
        np.testing.assert_allclose(rhs, -1j * psi, atol=1e-14)
    else:
        assert np.abs(rhs).max() == 0.0
        out = o.run(psi, 5)
        assert np.abs(out - 1).max() == 0.0


@pytest.mark.parametrize("scheme,pname", [("euler", "euler"), ("rk2", "rk2"), ("rk4", "rk4")])
@pytest.mark.parametrize("real_time", [True, False])
def test_linear_mode_amplification(scheme, pname, real_time):
    # eqn 4 with g = V = mu = 0 is psi_t = (i/2) lap psi: a Fourier mode
    # psi_k is multiplied by R(z), z = dt * (i/2) * lambda_k, per step.
    rp = rp_small(scheme=scheme, real_time=real_time, tau=0.01)
    o = Oracle(rp)
    X, Y, Z, d = mesh(o)
    k = [2 * np.pi * 2 / (rp.nx * d[0]), 2 * np.pi * 1 / (rp.ny * d[1]), 2 * np.pi * 1 / (rp.nz * d[2])]
    lam = sum(symbol(rp.order, kk, h) for kk, h in zip(k, d))
    psi0 = np.exp(1j * (k[0] * X + k[1] * Y + k[2] * Z)) * np.ones(o.shape)
    dt = rp.tau if real_time else -1j * rp.tau
    z = dt * 0.5j * lam
    out = o.run(psi0, 3)
    np.testing.assert_allclose(out, poly(pname, z) ** 3 * psi0, rtol=0, atol=1e-13)
    assert o.clock.p == 3
    if real_time:
        assert o.clock.t == pytest.approx(3 * rp.tau) and o.clock.im_t == 0.0
    else:
        assert o.clock.t == 0.0 and o.clock.im_t == pytest.approx(3 * rp.tau)


def test_cash_karp_tableau_identities():
    assert POLYS["ck_row_sums"] == ["0", "1/5", "3/10", "3/5", "1", "7/8"]
    assert POLYS["ck_sum_c"] == "1" and POLYS["ck_sum_cstar"] == "1"
    # the 5th-order solution matches exp(z) to z^5
    assert POLYS["ck5"][:6] == ["1", "1", "1/2", "1/6", "1/24", "1/120"]


def test_rkqs_linear_mode_and_step_control():
    # one accepted rkqs step on a Fourier mode: psi *= R_ck5(z); the error
    # norm is max|E(z) psi / psi_scal| / eps with psi_scal = |psi| + dt|f| + 1e-30.
    rp = rp_small(scheme="rk45", tau=0.01)
    o = Oracle(rp)
    X, Y, Z, d = mesh(o)
    k = [2 * np.pi * 1 / (rp.nx * d[0]), 0.0, 0.0]
    lam = symbol(rp.order, k[0], d[0])
    psi0 = np.exp(1j * k[0] * X) * np.ones(o.shape)
    out = o.run(psi0, 1)
    z = rp.tau * 0.5j * lam
    np.testing.assert_allclose(out, poly("ck5", z) * psi0, rtol=0, atol=1e-13)
    f = abs(0.5 * lam)
    err = abs(poly("ck_err", z)) / ((1.0 + rp.tau * f) + 1e-30) / 1e-6
    assert o.clock.errmax == pytest.approx(err, rel=1e-6)
    # step growth (solve.f90:214-220): errcon = (5/0.9)^(-5)
    errcon = (5 / 0.9) ** (1 / -0.2)
    grow = 0.9 * err ** -0.2 if err > errcon else 5.0
    assert o.clock.dt_re == pytest.approx(rp.tau * grow, rel=1e-12)
    assert o.clock.t == pytest.approx(rp.tau)


def test_rkqs_rejects_and_shrinks():
    # a stiff mode forces rejections: every retry shrinks dt by
    # max(0.9 errmax^-0.25, 0.1) (solve.f90:195-201); the accepted step
    # then satisfies errmax <= 1.
    rp = rp_small(scheme="rk45", tau=0.5, order=2)
    o = Oracle(rp)
    X, Y, Z, d = mesh(o)
    kx = 2 * np.pi * 4 / (rp.nx * d[0])
    psi0 = np.exp(1j * kx * X) * np.ones(o.shape)
    o.run(psi0, 1)
    assert o.clock.rejected >= 1
    assert o.clock.errmax <= 1.0
    assert 0 < o.clock.t < rp.tau


def test_norm_quadrature_exact_on_cubics():
    rp = rp_small(nx=11, ny=9, nz=7, xr=2.0, yr=1.5, zr=1.0)
    o = Oracle(rp)
    X, Y, Z, d = mesh(o)
    one = np.ones(o.shape, np.complex128)
    assert o.get_norm(one) == pytest.approx(8 * rp.xr * rp.yr * rp.zr, rel=1e-14)
    # |psi|^2 = 1 + x^2 -> integral = V + (2 xr^3/3)(2 yr)(2 zr)
    psi = np.sqrt(1 + X * X) * one
    exact = 8 * rp.xr * rp.yr * rp.zr + (2 * rp.xr ** 3 / 3) * (2 * rp.yr) * (2 * rp.zr)
    assert o.get_norm(psi) == pytest.approx(exact, rel=1e-13)


def test_energy_of_plane_wave():
    rp = rp_small(order=4, bcs=1)
    o = Oracle(rp)
    X, Y, Z, d = mesh(o)
    kx = 2 * np.pi * 2 / (rp.nx * d[0])
    A = 0.7
    psi = A * np.exp(1j * kx * X) * np.ones(o.shape)
    lam = symbol(4, kx, d[0])
    exact = rp.nx * rp.ny * rp.nz * (-lam * A * A + 0.5 * A ** 4) * d[0] * d[1] * d[2]
    assert o.energy(psi) == pytest.approx(exact, rel=1e-12)


def test_renormalise():
    rp = rp_small(nn=2.0)
    o = Oracle(rp)
    psi = np.full(o.shape, 1.5 + 0.5j)
    n = o.get_norm(psi)
    out = o.renormalise(psi, n)
    assert o.get_norm(out) == pytest.approx(2.0, rel=1e-14)


def test_ring_ic_matches_pade_profile():
    # BASELINE's ring: amplitude sqrt(d^2(0.3437+0.0286d^2)/(1+0.3333d^2+0.0286d^4))
    rp = RunParams(nx=32, ny=32, nz=32, xr=7.75, yr=7.75, zr=7.75)
    o = Oracle(rp)
    d = np.linspace(0, 6, 50)
    R = np.sqrt(d ** 2 * (0.3437 + 0.0286 * d ** 2) / (1 + 0.3333 * d ** 2 + 0.0286 * d ** 4))
    np.testing.assert_allclose(d * Oracle.get_rr(d), R, rtol=1e-14)
    ring = o.vortex_ring("xy", 0, 0, 0, 4.0, 0.0, 0, 0.0, 0, 1.0)
    np.testing.assert_allclose(ring, ic.vortex_ring(rp, "xy", r0=4.0), rtol=0, atol=1e-14)
    # far from the core |psi| -> 1
    assert abs(abs(ring[0, 0, 0]) - 1) < 0.02


@pytest.mark.parametrize("plane", ["xy", "xz", "yz"])
def test_product_ring_ic_matches_oracle(plane):
    rp = RunParams(nx=20, ny=18, nz=16, xr=6.0, yr=5.0, zr=4.0, scal=1.2)
    o = Oracle(rp)
    a = o.vortex_ring(plane, 0.5, -0.3, 0.2, 3.0, 0.2, 2, 0.3, 3, -1.0)
    b = ic.vortex_ring(rp, plane, 0.5, -0.3, 0.2, 3.0, 0.2, 2, 0.3, 3, -1.0)
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-13)


@pytest.mark.parametrize("dirn", ["x", "y", "z"])
def test_product_line_ics_match_oracle(dirn):
    rp = RunParams(nx=14, ny=12, nz=10, xr=4.0, yr=3.0, zr=2.5, mu=10.0, g=1.0, omx=0.1, omy=0.2, omz=0.3)
    o = Oracle(rp)
    kw = dict(x0=0.3, y0=-0.2, z0=0.1, amp1=0.2, amp2=0.1, ll=2.0, sgn=-1.0, dir=dirn)
    np.testing.assert_allclose(o.vortex_line(**kw), ic.vortex_line(rp, **kw), atol=1e-13)
    np.testing.assert_allclose(o.vortex_line(pade=True, **kw), ic.vortex_line_pade(rp, **kw), atol=1e-13)
    np.testing.assert_allclose(o.fermi(), ic.fermi(rp), atol=1e-13)


@pytest.mark.parametrize("kind", ["pulse", "ring"])
def test_pade_pulse_ring_ic(kind):
    # pade_pulse_ring (src/ic.f90:518-587): the oracle and the host
    # restatement agree; known answers of the closed form: psi = 1 where
    # x = x0 and s = r0 (the numerators carry the factor x2 + (1 - 2U^2) s2),
    # psi(x0 - d) = conj(psi(x0 + d)) (uu even and vv odd in x - x0), and
    # psi -> 1 far from the centre (along the axis vv -> -m/x^2 from above).
    rp = RunParams(nx=21, ny=21, nz=41, xr=10.0, yr=10.0, zr=20.0)  # unit spacing: x = 0 and s = 2 are nodes
    o = Oracle(rp)
    a = o.pade_pulse_ring(kind, 0.0, 0.0, 0.0, 2.0 if kind == "ring" else 0.0)
    b = ic.pade_pulse_ring(rp, kind, 0.0, 0.0, 0.0, 2.0 if kind == "ring" else 0.0)
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-14)
    j0 = 10 + (2 if kind == "ring" else 0)
    assert a[20, j0, 10] == 1.0 + 0.0j  # (x, y, z) = (0, s, 0) with s = r0
    np.testing.assert_allclose(a[:, :, ::-1], np.conj(a), rtol=0, atol=1e-15)
    m = 8.37 if kind == "pulse" else 8.97
    far = o.pade_pulse_ring(kind, -40.0, 0.0, 0.0, 0.0)[20, 10, 20]  # on the axis, 40 from the centre
    assert abs(far - 1.0) < 1e-2 and -m / 40.0 ** 2 < far.imag < -0.5 * m / 40.0 ** 2
    # off-centre arguments through both restatements
    kw = dict(x0=0.7, y0=-1.3, z0=2.1, r0=3.5)
    np.testing.assert_allclose(o.pade_pulse_ring(kind, **kw), ic.pade_pulse_ring(rp, kind, **kw), rtol=0, atol=1e-14)


def test_pair_sphere_wall_ics():
    # vortex_pair (src/ic.f90:591-636), sphere (:640-662), sphere2 (:666-684)
    # and wall (:688-709): oracle against the host restatement, and the
    # closed forms' known values.
    rp = RunParams(nx=21, ny=17, nz=81, xr=10.0, yr=8.0, zr=40.0)
    o = Oracle(rp)
    pair = o.vortex_pair()
    np.testing.assert_allclose(pair, ic.vortex_pair(rp), rtol=0, atol=1e-14)
    assert np.array_equal(pair, np.broadcast_to(pair[:1], pair.shape))  # the same in every z plane
    assert pair[0, 8, 10] == pytest.approx(1.0 - 1.14026, abs=1e-15)  # x = y = 0: 1 + a0, v = 0
    np.testing.assert_allclose(pair[:, :, ::-1], np.conj(pair), rtol=0, atol=1e-15)
    sph = o.sphere()
    np.testing.assert_allclose(sph, ic.sphere(rp), rtol=0, atol=1e-14)
    assert sph[40, 8, 10].real == pytest.approx(0.5 * (1.0 + np.tanh(-12.0)), rel=1e-14)
    sph2 = o.sphere2()
    np.testing.assert_allclose(sph2, ic.sphere2(rp), rtol=1e-14, atol=0)
    assert sph2[40, 8, 10] == 100.0
    w = o.wall()
    np.testing.assert_array_equal(w, ic.wall(rp))
    zc = np.linspace(-40.0, 40.0, 81)
    np.testing.assert_array_equal(w[:, 0, 0].real, np.where(zc <= -30.0, 0.0, 1.0))


def test_golden_oracle_regression():
    """The oracle still reproduces its committed small-grid runs bit for bit."""
    from tests.golden.make_golden import CASES, SHAPE

    z = np.load(GOLD / "oracle_small.npz")
    for name, kw, steps in CASES:
        rp = RunParams(**SHAPE, **kw)
        o = Oracle(rp)
        psi = o.run(z[f"{name}/psi0"], int(z[f"{name}/steps"]))
        np.testing.assert_array_equal(psi, z[f"{name}/psi"], err_msg=name)
        assert o.get_norm(psi) == float(z[f"{name}/norm"])
        assert o.energy(psi) == float(z[f"{name}/energy"])
