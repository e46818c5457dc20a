"""The C-ABI library loads without a GPU, exports every entry point that
include/*.h declares, validates arguments, and has no CPU fallback."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from gpe_b200 import _lib as L
from gpe_b200.solver import RunParams

ROOT = Path(__file__).resolve().parents[1]


def declared_in_headers() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(gpe_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_headers_declare_entry_points():
    names = declared_in_headers()
    assert {"gpe_create", "gpe_step", "gpe_norm", "gpe_energy", "gpe_destroy"} <= names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = declared_in_headers() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    for name in declared_in_headers():
        assert hasattr(lib, name)


def test_ctypes_prototypes_cover_header():
    assert declared_in_headers() <= set(L.declared_symbols()) | set(getattr(L, "EXTRA_SYMBOLS", []))


def test_param_validation_without_gpu():
    lib = L.load()
    ok = RunParams(nx=64, ny=64, nz=64).to_c()
    assert lib.gpe_state_bytes(C.byref(ok)) > 0
    for bad in (dict(nx=4), dict(order=3), dict(bcs=0), dict(eqn_to_solve=5), dict(tau=0.0)):
        p = RunParams(**bad).to_c()
        assert lib.gpe_state_bytes(C.byref(p)) == -1
        h = C.c_void_p()
        assert lib.gpe_create(C.byref(p), C.byref(h)) == L.GPE_ERR_BADARG
        assert lib.gpe_last_error(None)
    p = RunParams().to_c()
    p.scheme = 9
    h = C.c_void_p()
    assert lib.gpe_create(C.byref(p), C.byref(h)) == L.GPE_ERR_BADARG
    assert b"Unrecognised time stepping scheme" in lib.gpe_last_error(None)


def test_state_bytes_layout():
    # 256^3 complex128 RK4: 4 ghost-padded fields
    lib = L.load()
    p = RunParams(nx=256, ny=256, nz=256, scheme="rk4").to_c()
    px = ((8 + 256 + 2) + 7) // 8 * 8
    assert lib.gpe_state_bytes(C.byref(p)) == 4 * 16 * px * 260 * 260
    p = RunParams(nx=256, ny=256, nz=256, scheme="rk4", storage="c64").to_c()
    px = ((16 + 256 + 2) + 15) // 16 * 16
    assert lib.gpe_state_bytes(C.byref(p)) == 4 * 8 * px * 260 * 260


def test_no_cpu_fallback_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    lib = L.load()
    p = RunParams(nx=16, ny=16, nz=16).to_c()
    h = C.c_void_p()
    rc = lib.gpe_create(C.byref(p), C.byref(h))
    assert rc == L.GPE_ERR_CUDA
    assert not h.value


def test_norm_noalloc_rejects_misaligned_pointers_before_any_launch():
    """gpe_norm_noalloc checks its caller-owned pointers for the alignment its
    kernels load and store with, and returns GPE_ERR_BADARG without touching
    the device (these addresses are never dereferenced: the call is rejected
    before any CUDA call, which also holds without a GPU)."""
    lib = L.load()
    args = (6, 6, 6, 1.0, 1.0, 1.0)
    good = 0x10000
    # complex128 input must be 16-byte aligned
    assert lib.gpe_norm_noalloc(C.c_void_p(good + 8), L.GPE_C128, *args, C.c_void_p(good), None) == L.GPE_ERR_BADARG
    # complex64 input 8-byte aligned
    assert lib.gpe_norm_noalloc(C.c_void_p(good + 4), L.GPE_C64, *args, C.c_void_p(good), None) == L.GPE_ERR_BADARG
    # the output double 8-byte aligned
    assert lib.gpe_norm_noalloc(C.c_void_p(good), L.GPE_C64, *args, C.c_void_p(good + 4), None) == L.GPE_ERR_BADARG
    # size limit and dtype, also before any CUDA call
    assert lib.gpe_norm_noalloc(C.c_void_p(good), L.GPE_C128, 6, 6, L.GPE_NOALLOC_MAX_NZ + 1, 1.0, 1.0, 1.0,
                                C.c_void_p(good), None) == L.GPE_ERR_BADARG
    assert lib.gpe_norm_noalloc(C.c_void_p(good), 7, *args, C.c_void_p(good), None) == L.GPE_ERR_BADARG
