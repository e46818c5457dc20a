"""gpe_norm_noalloc: the allocation-free norm for callers that own every
byte of device memory (a framework allocator, a fixed budget, a loop that
must not allocate between steps).  The caller hands in its own device input
and output buffers; the library uses only its built-in scratch array.

Checked through the C ABI against the existing gpe_norm on the same state,
on two calls in a row (the second call reuses the shared scratch left by the
first), for complex128 and complex64 data, plus the size limit.  This file
is collected last so that a failure here never hides another test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # same bound as the other norm comparisons


@pytest.mark.parametrize("storage", ["c128", "c64"])
def test_norm_noalloc_matches_gpe_norm(gpu, storage):
    import torch

    from gpe_b200 import _lib as L
    from gpe_b200 import ic
    from gpe_b200.solver import RunParams, Solver

    lib = L.load()
    rp = RunParams(nx=40, ny=36, nz=30, xr=9.75, yr=8.75, zr=7.25, bcs=2, order=4, storage=storage)
    psi = ic.vortex_ring(rp, "xy", r0=3.0)
    rng = np.random.default_rng(21)
    psi = psi + 0.1 * (rng.standard_normal(psi.shape) + 1j * rng.standard_normal(psi.shape))
    if storage == "c64":
        psi = psi.astype(np.complex64)
    code = L.GPE_C64 if storage == "c64" else L.GPE_C128
    s = Solver(rp)
    s.set_state(psi)
    ref = s.get_norm()
    _, _, _, d = s.grid()
    # caller-owned device buffers
    d_psi = torch.from_numpy(np.ascontiguousarray(psi)).cuda()
    d_out = torch.empty(1, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        d_out.fill_(-1.0)
        rc = lib.gpe_norm_noalloc(C.c_void_p(d_psi.data_ptr()), code, rp.nx, rp.ny, rp.nz, d[0], d[1], d[2],
                                  C.c_void_p(d_out.data_ptr()), stream)
        assert rc == L.GPE_OK
        torch.cuda.synchronize()
        assert d_out.item() == pytest.approx(ref, rel=TOL)
    s.close()


def test_norm_noalloc_rejects_oversize(gpu):
    import torch

    from gpe_b200 import _lib as L

    lib = L.load()
    buf = torch.empty(2, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = lib.gpe_norm_noalloc(p, L.GPE_C128, 8, 8, 8193, 1.0, 1.0, 1.0, p, None)
    assert rc == L.GPE_ERR_BADARG
