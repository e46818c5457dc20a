"""The thread layouts of the complex64 stage kernel give identical results.

With complex64 storage and the FP32 stencil the stage kernel runs by default
with two x-adjacent sites per thread (16-byte shared-memory reads and
stores, 32 x 16 tiles); the one-site-per-column layout (32 x 8 tiles) does
the same per-site arithmetic, so the states must agree bit for bit, on grids
whose x extent is odd (a pair's second site outside the grid), whose y
extent is not a multiple of the tile height, for both orders and boundary
conditions, every scheme, and the fused norm and energy.  The layout is
chosen at handle creation through GPE_TILE.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from gpe_b200 import ic
from gpe_b200.solver import RunParams, Solver
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

LAYOUTS = {"row2": "4", "pair_32x8": "16", "pair_32x16": "32"}


def run_with(layout, rp, psi0, steps, **kw):
    old = os.environ.get("GPE_TILE")
    os.environ["GPE_TILE"] = LAYOUTS[layout]
    try:
        s = Solver(rp)
    finally:
        if old is None:
            del os.environ["GPE_TILE"]
        else:
            os.environ["GPE_TILE"] = old
    s.set_state(psi0)
    info = s.solver(steps, **kw)
    out = s.get_state(np.complex64)
    e = s.energy()
    s.close()
    return out, info, e


@pytest.mark.parametrize("shape", [(37, 21, 19), (64, 40, 23), (7, 17, 9), (33, 6, 7)])
@pytest.mark.parametrize("order,bcs", [(2, 1), (2, 2), (4, 1), (4, 2)])
@pytest.mark.parametrize("scheme", ["euler", "rk2", "rk4", "rk45"])
def test_pair_layouts_equal_row_layout_bitwise(gpu, shape, order, bcs, scheme):
    nx, ny, nz = shape
    rp = RunParams(nx=nx, ny=ny, nz=nz, xr=0.5 * (nx - 1), yr=0.5 * (ny - 1), zr=0.5 * (nz - 1), tau=0.004,
                   scheme=scheme, eqn_to_solve=4, bcs=bcs, order=order, g=1.0, mu=2.0, omx=0.3, omy=0.2, omz=0.25,
                   storage="c64", compute="f32")
    rng = np.random.default_rng(nx * 131 + ny * 7 + nz + order + bcs)
    psi0 = (1.0 + 0.2 * (rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx)))).astype(np.complex64)
    ref, iref, eref = run_with("row2", rp, psi0, 6, want_norm=True, want_energy=True)
    for layout in ("pair_32x8", "pair_32x16"):
        out, info, e = run_with(layout, rp, psi0, 6, want_norm=True, want_energy=True)
        np.testing.assert_array_equal(out, ref)
        # the per-CTA partial sums follow the tile shape, so the reductions
        # are the same sums in another order
        assert info.norm == pytest.approx(iref.norm, rel=1e-13)
        assert info.energy == pytest.approx(iref.energy, rel=1e-13) and e == pytest.approx(eref, rel=1e-13)
        assert (info.dt_re, info.dt_im, info.t) == (iref.dt_re, iref.dt_im, iref.t)


@pytest.mark.parametrize("eqn", [1, 2, 3])
def test_pair_layout_other_equations_with_urhs_and_diss(gpu, eqn):
    rp = RunParams(nx=45, ny=35, nz=21, xr=5.5, yr=4.25, zr=2.5, tau=0.003, scheme="rk4", eqn_to_solve=eqn,
                   bcs=1, order=4, Urhs=0.2, diss_amp=0.1 if eqn != 2 else 0.0, storage="c64", compute="f32")
    rng = np.random.default_rng(eqn)
    psi0 = (1.0 + 0.3 * (rng.normal(size=(21, 35, 45)) + 1j * rng.normal(size=(21, 35, 45)))).astype(np.complex64)
    ref, _, _ = run_with("row2", rp, psi0, 5)
    out, _, _ = run_with("pair_32x16", rp, psi0, 5)
    np.testing.assert_array_equal(out, ref)
    # and the layout is within the FP32 bar of the FP64 oracle
    o = Oracle(rp.replace(storage="c128", compute="auto")).run(psi0.astype(np.complex128), 5)
    assert float(np.linalg.norm((out - o).ravel()) / np.linalg.norm(o.ravel())) <= 1e-5
