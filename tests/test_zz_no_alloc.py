"""gpe_norm_noalloc: the allocation-free norm for callers that own every
byte of device memory (a framework allocator, a fixed budget, a loop that
must not allocate between steps).  The caller hands in its own device input
and output buffers; the library uses only its built-in scratch array.

Checked through the C ABI against the existing gpe_norm on the same state,
on two calls in a row (the second call reuses the shared scratch left by the
first), for complex128 and complex64 data, on grids whose plane count runs
past one reduction block (300 planes) and up to the documented limit, plus
the size limit and a check that repeated calls leave the device's free
memory unchanged.  This file is collected last so that a failure here never
hides another test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # same bound as the other norm comparisons


def _noalloc_norm(lib, L, d_psi, code, rp, d, d_out, stream):
    d_out.fill_(-1.0)
    rc = lib.gpe_norm_noalloc(C.c_void_p(d_psi.data_ptr()), code, rp.nx, rp.ny, rp.nz, d[0], d[1], d[2],
                              C.c_void_p(d_out.data_ptr()), stream)
    assert rc == L.GPE_OK
    return rc


@pytest.mark.parametrize("storage", ["c128", "c64"])
@pytest.mark.parametrize("shape", [(40, 36, 30), (8, 8, 300), (6, 6, 8192)])
def test_norm_noalloc_matches_gpe_norm(gpu, storage, shape):
    import torch

    from gpe_b200 import _lib as L
    from gpe_b200.solver import RunParams, Solver

    lib = L.load()
    nx, ny, nz = shape
    rp = RunParams(nx=nx, ny=ny, nz=nz, xr=0.25 * (nx - 1), yr=0.25 * (ny - 1), zr=0.25 * (nz - 1), bcs=2,
                   order=4, storage=storage)
    rng = np.random.default_rng(21 + nz)
    psi = 1.0 + 0.3 * (rng.standard_normal((nz, ny, nx)) + 1j * rng.standard_normal((nz, ny, nx)))
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
        _noalloc_norm(lib, L, d_psi, code, rp, d, d_out, stream)
        torch.cuda.synchronize()
        assert d_out.item() == pytest.approx(ref, rel=TOL)
    s.close()


def test_norm_noalloc_allocates_nothing(gpu):
    """After a first call, further calls leave the device's free memory as it
    was: the scratch is the library's static array."""
    import torch

    from gpe_b200 import _lib as L
    from gpe_b200.solver import RunParams

    lib = L.load()
    rp = RunParams(nx=48, ny=40, nz=320, xr=5.0, yr=5.0, zr=5.0)
    d = (2 * rp.xr / (rp.nx - 1), 2 * rp.yr / (rp.ny - 1), 2 * rp.zr / (rp.nz - 1))
    d_psi = torch.ones((rp.nz, rp.ny, rp.nx), dtype=torch.complex128, device="cuda")
    d_out = torch.empty(1, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _noalloc_norm(lib, L, d_psi, L.GPE_C128, rp, d, d_out, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(20):
        _noalloc_norm(lib, L, d_psi, L.GPE_C128, rp, d, d_out, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.isfinite(d_out.item()) and d_out.item() > 0


def test_norm_noalloc_rejects_oversize(gpu):
    import torch

    from gpe_b200 import _lib as L

    lib = L.load()
    buf = torch.empty(2, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = lib.gpe_norm_noalloc(p, L.GPE_C128, 8, 8, L.GPE_NOALLOC_MAX_NZ + 1, 1.0, 1.0, 1.0, p, None)
    assert rc == L.GPE_ERR_BADARG
