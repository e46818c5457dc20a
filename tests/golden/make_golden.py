"""Generate the committed known-answer fixtures under tests/golden/.

    python tests/golden/make_golden.py

kat_polys.json   -- exact (rational) amplification polynomials of the
                    reference's time integrators applied to y' = z y, derived
                    from the Butcher tableaux written in src/solve.f90
                    (Euler :68, RK2 :91-99, RK4 :124-148, Cash-Karp :255-281).
                    These are analytic facts of the reference's algorithm,
                    independent of any implementation here.
oracle_small.npz -- small-grid runs of the CPU oracle (regression pins for
                    the oracle and direct fixtures for GPU parity): initial
                    state, state after a few solver() calls, norm, energy.
"""
from __future__ import annotations

import json
import sys
from fractions import Fraction as F
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

# Cash-Karp tableau exactly as typed in src/solve.f90:255-281
CK_A = [
    [],
    [F(1, 5)],
    [F(3, 40), F(9, 40)],
    [F(3, 10), F(-9, 10), F(6, 5)],
    [F(-11, 54), F(5, 2), F(-70, 27), F(35, 27)],
    [F(1631, 55296), F(175, 512), F(575, 13824), F(44275, 110592), F(253, 4096)],
]
CK_C = [F(37, 378), F(0), F(250, 621), F(125, 594), F(0), F(512, 1771)]
CK_CS = [F(2825, 27648), F(0), F(18575, 48384), F(13525, 55296), F(277, 14336), F(1, 4)]


def explicit_poly(A, b):
    """Coefficients of R(z) = 1 + z b^T (I - zA)^{-1} 1 for explicit A."""
    s = len(b)
    # u_k = A^k 1
    u = [F(1)] * s
    coeffs = [F(1)]
    for k in range(s):
        coeffs.append(sum(bi * ui for bi, ui in zip(b, u)))
        u = [sum((A[i][j] if j < len(A[i]) else F(0)) * u[j] for j in range(s)) for i in range(s)]
    while len(coeffs) > 1 and coeffs[-1] == 0:
        coeffs.pop()
    return coeffs


def polys():
    euler = explicit_poly([[]], [F(1)])
    rk2 = explicit_poly([[], [F(1, 2)]], [F(0), F(1)])
    rk4 = explicit_poly([[], [F(1, 2)], [F(0), F(1, 2)], [F(0), F(0), F(1)]],
                        [F(1, 6), F(1, 3), F(1, 3), F(1, 6)])
    ck5 = explicit_poly(CK_A, CK_C)
    dc = [c - cs for c, cs in zip(CK_C, CK_CS)]
    ck_err = explicit_poly(CK_A, dc)
    ck_err[0] = F(0)  # the error estimate has no constant term
    row_sums = [str(sum(r, F(0))) for r in CK_A]
    return {
        "euler": [str(c) for c in euler],
        "rk2": [str(c) for c in rk2],
        "rk4": [str(c) for c in rk4],
        "ck5": [str(c) for c in ck5],
        "ck_err": [str(c) for c in ck_err],
        "ck_row_sums": row_sums,
        "ck_sum_c": str(sum(CK_C)),
        "ck_sum_cstar": str(sum(CK_CS)),
    }


CASES = [
    # name, params, steps
    ("rk4_eq4_refl_o2", dict(scheme="rk4", eqn_to_solve=4, bcs=2, order=2, g=1.0, mu=1.0), 6),
    ("rk4_eq4_per_o4", dict(scheme="rk4", eqn_to_solve=4, bcs=1, order=4, g=1.0, mu=1.0, omx=0.3, omy=0.2, omz=0.1), 6),
    ("rk4_eq1_refl_o4_diss", dict(scheme="rk4", eqn_to_solve=1, bcs=2, order=4, diss_amp=0.1, Urhs=0.3), 6),
    ("rk4_eq2_per_o2_urhs", dict(scheme="rk4", eqn_to_solve=2, bcs=1, order=2, Urhs=0.2), 6),
    ("rk4_eq3_refl_o2", dict(scheme="rk4", eqn_to_solve=3, bcs=2, order=2, diss_amp=0.05), 6),
    ("euler_eq4_per_o4", dict(scheme="euler", eqn_to_solve=4, bcs=1, order=4, g=2.0, mu=0.5), 6),
    ("rk2_eq1_per_o4", dict(scheme="rk2", eqn_to_solve=1, bcs=1, order=4), 6),
    ("rk45_eq4_refl_o4", dict(scheme="rk45", eqn_to_solve=4, bcs=2, order=4, g=1.0, mu=2.0, omx=0.2, omy=0.2, omz=0.1), 4),
    ("rk4_eq4_imag_refl_o2", dict(scheme="rk4", eqn_to_solve=4, bcs=2, order=2, real_time=False, g=1.0, mu=1.0, omx=0.5, omy=0.5, omz=0.5), 6),
    ("rk4_eq4_gamma_refl_o4", dict(scheme="rk4", eqn_to_solve=4, bcs=2, order=4, g=1.0, mu=1.0, gamma=0.05, omx=0.1, omy=0.1, omz=0.1), 6),
]
SHAPE = dict(nx=13, ny=11, nz=9, xr=3.0, yr=2.5, zr=2.0, tau=0.002)


def initial_state(shape, seed):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    z = np.linspace(-1, 1, nz)[:, None, None]
    y = np.linspace(-1, 1, ny)[None, :, None]
    x = np.linspace(-1, 1, nx)[None, None, :]
    base = np.exp(-(x * x + 2 * y * y + 3 * z * z)) * np.exp(1j * (x + 0.5 * y * z))
    noise = 0.05 * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    return np.ascontiguousarray(base + noise, dtype=np.complex128)


def oracle_cases():
    from gpe_b200.solver import RunParams
    from oracle.pyoracle import Oracle

    out = {}
    for n, (name, kw, steps) in enumerate(CASES):
        rp = RunParams(**SHAPE, **kw)
        o = Oracle(rp)
        psi0 = initial_state((rp.nz, rp.ny, rp.nx), 100 + n)
        psi = o.run(psi0, steps)
        out[f"{name}/psi0"] = psi0
        out[f"{name}/psi"] = psi
        out[f"{name}/steps"] = np.array(steps)
        out[f"{name}/clock"] = np.array([o.clock.t, o.clock.im_t, o.clock.dt_re, o.clock.dt_im])
        out[f"{name}/norm"] = np.array(o.get_norm(psi))
        out[f"{name}/energy"] = np.array(o.energy(psi))
    return out


def main():
    (HERE / "kat_polys.json").write_text(json.dumps(polys(), indent=1) + "\n")
    np.savez_compressed(HERE / "oracle_small.npz", **oracle_cases())
    print("wrote", HERE / "kat_polys.json", HERE / "oracle_small.npz")


if __name__ == "__main__":
    main()
