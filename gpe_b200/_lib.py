"""ctypes binding of libgpe_cuda.so (include/gpe_cuda.h).

The library is loaded from this package's lib/ directory only; there is no
fallback implementation.  If the shared object is missing the import of the
solver fails loudly with instructions to build it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# GPE_CUDA_LIB selects another build of the library (default: the in-tree one)
LIB_PATH = Path(os.environ.get("GPE_CUDA_LIB") or Path(__file__).resolve().parent / "lib" / "libgpe_cuda.so")

GPE_OK = 0
GPE_ERR_BADARG = -1
GPE_ERR_CUDA = -2
GPE_ERR_NONFINITE = -3
GPE_ERR_TIMEOUT = -4
GPE_ERR_NOMEM = -5
GPE_ERR_NOMEM_BUDGET = -6
GPE_ERR_STATE = -7

GPE_EULER, GPE_RK2, GPE_RK4, GPE_RK45 = 0, 1, 2, 3
GPE_C128, GPE_C64 = 0, 1
GPE_COMPUTE_AUTO, GPE_COMPUTE_F32, GPE_COMPUTE_F64 = 0, 1, 2

# planes of built-in scratch in gpe_norm_noalloc (include/gpe_cuda.h)
GPE_NOALLOC_MAX_NZ = 8192

SCHEMES = {"euler": GPE_EULER, "rk2": GPE_RK2, "rk4": GPE_RK4, "rk45": GPE_RK45}


class GpeParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("scheme", C.c_int32), ("eqn", C.c_int32), ("bcs", C.c_int32), ("order", C.c_int32),
        ("real_time", C.c_int32), ("storage", C.c_int32), ("compute", C.c_int32),
        ("tile_zc", C.c_int32), ("reserved", C.c_int32),
        ("xr", C.c_double), ("yr", C.c_double), ("zr", C.c_double),
        ("tau", C.c_double),
        ("Urhs", C.c_double), ("diss_amp", C.c_double), ("scal", C.c_double), ("g", C.c_double),
        ("mu", C.c_double), ("nn", C.c_double), ("omx", C.c_double), ("omy", C.c_double),
        ("omz", C.c_double), ("gamma", C.c_double),
        ("eps", C.c_double), ("safety", C.c_double), ("dt_decrease", C.c_double),
        ("dt_increase", C.c_double),
    ]


class GpeStepInfo(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("im_t", C.c_double), ("dt_re", C.c_double), ("dt_im", C.c_double),
        ("p", C.c_int64), ("accepted", C.c_int64), ("rejected", C.c_int64),
        ("errmax", C.c_double), ("norm", C.c_double), ("energy", C.c_double),
        ("want_norm", C.c_int32), ("want_energy", C.c_int32),
    ]


(GPE_IC_UNIFORM, GPE_IC_FERMI, GPE_IC_LINE, GPE_IC_RING, GPE_IC_LINE_PADE, GPE_IC_RANDOM_PHASE, GPE_IC_PADE_PULSE,
 GPE_IC_PADE_RING, GPE_IC_VORTEX_PAIR, GPE_IC_SPHERE, GPE_IC_SPHERE2, GPE_IC_WALL) = range(12)


class GpeRing(C.Structure):
    _fields_ = [("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("r0", C.c_double),
                ("amp", C.c_double), ("r1", C.c_double), ("dir", C.c_double), ("mm", C.c_int32),
                ("kk", C.c_int32), ("plane", C.c_char * 4), ("reserved", C.c_int32)]


class GpeLine(C.Structure):
    _fields_ = [("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("amp1", C.c_double),
                ("amp2", C.c_double), ("ll", C.c_double), ("sgn", C.c_double), ("imprint_phase", C.c_int32),
                ("dir", C.c_char), ("reserved", C.c_char * 3)]


class GpePulse(C.Structure):
    _fields_ = [("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("r0", C.c_double)]


class GpeIC(C.Structure):
    _fields_ = [("nfactors", C.c_int32), ("factor", C.c_int32 * 4), ("reserved", C.c_int32),
                ("ring", GpeRing), ("line", GpeLine), ("seed", C.c_uint64), ("kc", C.c_double),
                ("pulse", GpePulse)]


class GpeResult(C.Structure):
    _fields_ = [
        ("tag", C.c_uint64), ("status", C.c_int32), ("reserved", C.c_int32),
        ("steps", C.c_int64), ("rejected", C.c_int64),
        ("t", C.c_double), ("im_t", C.c_double), ("dt_re", C.c_double), ("dt_im", C.c_double),
        ("norm", C.c_double), ("submit_s", C.c_double), ("start_s", C.c_double), ("finish_s", C.c_double),
    ]


class GpeCondensedInfo(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("M", "n0", "rho0", "tot", "temp", "temp2", "H", "mass_density")]


GPE_SPECTRUM_SHELLS = 7

_PROTOS = {
    "gpe_create": (C.c_int, [C.POINTER(GpeParams), C.POINTER(C.c_void_p)]),
    "gpe_destroy": (None, [C.c_void_p]),
    "gpe_last_error": (C.c_char_p, [C.c_void_p]),
    "gpe_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "gpe_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "gpe_set_state_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "gpe_get_state_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "gpe_step": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(GpeStepInfo)]),
    "gpe_step_async": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(GpeStepInfo)]),
    "gpe_sync": (C.c_int, [C.c_void_p]),
    "gpe_norm": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "gpe_energy": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "gpe_renormalise": (C.c_int, [C.c_void_p, C.c_double]),
    "gpe_get_grid": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "gpe_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "gpe_state_bytes": (C.c_int64, [C.POINTER(GpeParams)]),
    "gpe_version": (C.c_char_p, []),
    "gpe_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "gpe_profile_get": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                  C.POINTER(C.c_double)]),
    "gpe_pool_create": (C.c_int, [C.c_int64, C.POINTER(C.c_void_p)]),
    "gpe_pool_submit": (C.c_int, [C.c_void_p, C.POINTER(GpeParams), C.c_void_p, C.c_int32, C.c_int64, C.c_uint64,
                                  C.c_void_p]),
    "gpe_pool_submit_ic": (C.c_int, [C.c_void_p, C.POINTER(GpeParams), C.POINTER(GpeIC), C.c_int64, C.c_uint64,
                                     C.c_void_p]),
    "gpe_set_ic": (C.c_int, [C.c_void_p, C.POINTER(GpeIC)]),
    "gpe_multiply_ic": (C.c_int, [C.c_void_p, C.POINTER(GpeIC), C.c_int32]),
    "gpe_condensed": (C.c_int, [C.c_void_p, C.POINTER(GpeCondensedInfo), C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_int32]),
    "gpe_filtered": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_int32]),
    "gpe_get_site": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    "gpe_snapshot_begin": (C.c_int, [C.c_void_p, C.c_int32]),
    "gpe_snapshot_wait": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "gpe_set_state_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "gpe_get_state_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "gpe_wait_copies": (C.c_int, [C.c_void_p]),
    "gpe_host_alloc": (C.c_void_p, [C.c_size_t]),
    "gpe_host_free": (None, [C.c_void_p]),
    "gpe_slab_nccl_id": (C.c_int, [C.c_void_p]),
    "gpe_slab_hub_create": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "gpe_slab_hub_destroy": (None, [C.c_void_p]),
    "gpe_create_slab": (C.c_int, [C.POINTER(GpeParams), C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                  C.POINTER(C.c_void_p)]),
    "gpe_slab_extent": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "gpe_slab_partition": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32)]),
    "gpe_pool_step": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int32)]),
    "gpe_pool_poll": (C.c_int, [C.c_void_p, C.POINTER(GpeResult), C.c_int32, C.POINTER(C.c_int32)]),
    "gpe_pool_free_bytes": (C.c_int64, [C.c_void_p]),
    "gpe_pool_solve_bytes": (C.c_int64, [C.POINTER(GpeParams)]),
    "gpe_pool_last_error": (C.c_char_p, [C.c_void_p]),
    "gpe_pool_destroy": (None, [C.c_void_p]),
    "gpe_test_expire_waits": (C.c_int, [C.c_void_p]),
    "gpe_pool_test_expire_waits": (C.c_int, [C.c_void_p]),
    "gpe_norm_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                   C.c_double, C.c_double, C.c_void_p, C.c_void_p]),
}

KIND_NAMES = ["euler", "rk2_1", "rk2_2", "rk4_1", "rk4_2", "rk4_4", "ck_1", "ck_2", "ck_3", "ck_4", "ck_5",
              "ck_6", "energy", "rk4_3"]

_lib = None


class GpeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gpe error {code}: {msg}")
        self.code = code


def load() -> C.CDLL:
    """Load libgpe_cuda.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library with `python -m gpe_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | C.RTLD_GLOBAL)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols() -> list[str]:
    return list(_PROTOS)


def pinned_empty(shape, dtype) -> "np.ndarray":
    """An uninitialised numpy array in page-locked host memory
    (gpe_host_alloc), freed when the array is garbage-collected."""
    import weakref

    import numpy as np

    lib = load()
    dt = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dt.itemsize
    ptr = lib.gpe_host_alloc(max(nbytes, 1))
    if not ptr:
        raise MemoryError("gpe_host_alloc failed")
    buf = (C.c_char * max(nbytes, 1)).from_address(ptr)
    weakref.finalize(buf, lib.gpe_host_free, ptr)
    return np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)
